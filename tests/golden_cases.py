"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import glob
import os

import numpy as np

from apollo_b200.mesh import Mesh

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "*.npz")))

BC_NAMES = {0: "gridFixedBC", 1: "isentropicVortexBC", 2: "maxwellTransverseMagneticBC", 3: "phmConductingWallBC"}


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    d = {k: z[k] for k in z.files}
    mesh = Mesh(vx=d["vx"], vy=d["vy"], etov=d["etov"], face_tag=d["face_tag"], vert_canon=d["vert_canon"], n=0,
                lo=(0, 0), hi=(1, 1), periodic=False)
    d["mesh"] = mesh
    d["equation"] = str(d["equation"])
    par = d.get("bc_params", np.zeros((len(d["bc_kinds"]), 0)))
    d["bcs"] = tuple((BC_NAMES[int(k)], tuple(par[i]) if par.shape[1] else ()) for i, k in enumerate(d["bc_kinds"]))
    return d


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)
