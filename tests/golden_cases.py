"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import glob
import os

import numpy as np

from apollo_b200.mesh import Mesh

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "*.npz")))

BC_NAMES = {0: "gridFixedBC", 1: "isentropicVortexBC", 2: "maxwellTransverseMagneticBC", 3: "phmConductingWallBC",
            4: "eulerWallBC", 5: "eulerInflowBC", 6: "eulerZeroGradientBC", 7: "eulerDirichletBC"}
# the parameters each kind takes, of the 8 stored per condition
BC_NPARAMS = {0: 1, 1: 6, 2: 0, 3: 0, 4: 0, 5: 5, 6: 0, 7: 6}


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    d = {k: z[k] for k in z.files}
    mesh = Mesh(vx=d["vx"], vy=d["vy"], etov=d["etov"], face_tag=d["face_tag"], vert_canon=d["vert_canon"], n=0,
                lo=(0, 0), hi=(1, 1), periodic=False)
    d["mesh"] = mesh
    d["equation"] = str(d["equation"])
    par = d.get("bc_params", np.zeros((len(d["bc_kinds"]), 8)))
    d["bcs"] = tuple((BC_NAMES[int(k)], tuple(par[i][:BC_NPARAMS[int(k)]])) for i, k in enumerate(d["bc_kinds"]))
    d["numflux"] = str(d["numflux"]) if "numflux" in d else "LF"
    d["sources"] = tuple((str(k), (int(o),), tuple(p[:n])) for k, o, p, n in
                         zip(d.get("src_kinds", ()), d.get("src_out", ()), d.get("src_params", ()),
                             d.get("src_nparams", ())))
    return d


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def is_lf(name):
    """Fixtures with the Lax-Friedrichs flux and no limiter (what the mixed and
    adjoint forms support)."""
    d = load(name)
    return d["numflux"] == "LF" and "limiter" not in d


LF_NAMES = [n for n in NAMES if is_lf(n)]
