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


def channel_mesh(n, seed, rotate_seed=None):
    """[0,2] x [0,1] channel: bottom wall (tag 1), right outflow (2), top
    inflow (3), left Dirichlet (4).  With ``rotate_seed`` each element's
    vertex list is rotated by a random shift (orientation kept, face tags
    follow), so boundary faces sit in every face slot, after interior faces
    too."""
    from apollo_b200.mesh import jittered_square
    mesh = jittered_square(n, (0.0, 0.0), (2.0, 1.0), seed=seed, periodic=False, wall_tag=1)
    for f, (i, j) in enumerate(((0, 1), (1, 2), (2, 0))):
        xa, ya = mesh.vx[mesh.etov[:, i]], mesh.vy[mesh.etov[:, i]]
        xb, yb = mesh.vx[mesh.etov[:, j]], mesh.vy[mesh.etov[:, j]]
        mesh.face_tag[:, f] = np.select([(ya == 0) & (yb == 0), (xa == 2) & (xb == 2), (ya == 1) & (yb == 1),
                                         (xa == 0) & (xb == 0)], [1, 2, 3, 4], 0)
    if rotate_seed is not None:
        shift = np.random.default_rng(rotate_seed).integers(0, 3, mesh.K)
        idx = (np.arange(3)[None, :] + shift[:, None]) % 3
        mesh.etov = np.ascontiguousarray(np.take_along_axis(mesh.etov, idx, axis=1))
        mesh.face_tag = np.ascontiguousarray(np.take_along_axis(mesh.face_tag, idx, axis=1))
    return mesh


CHANNEL_INFLOW = (0.4, -60.0, 1.4, 1.0, 1.0)      # Mach_number, Flow_angle, gas_gamma, Pressure, density
CHANNEL_DIRICHLET = (1.0, 0.5, 0.0, 0.0, 1.4, 1.0)  # density, x/y/zvelocity, gas_gamma, pressure


def channel_state(x, y, rough=0.0, seed=0):
    """Euler channel state (5 fields): density bump, transverse velocity wave,
    pressure variation, with a relative random perturbation ``rough``."""
    rho = 1.0 + 0.3 * np.exp(-((x - 1.0) ** 2 + (y - 0.5) ** 2) / 0.05)
    u, v, p = 0.5 + 0 * x, 0.2 * np.sin(np.pi * x), 1.0 + 0.5 * np.cos(2 * np.pi * y)
    U = np.stack([rho, rho * u, rho * v, 0 * x, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=-1)
    if rough:
        rng = np.random.default_rng(seed)
        U = U * (1.0 + rough * rng.standard_normal(U.shape))
        U[..., 3] = 0.3 * rough * rng.standard_normal(x.shape)
    return np.ascontiguousarray(U)


def boundary_after_interior(conn, N):
    """Elements whose boundary face at a position the Euler limiters read
    comes after an interior face (the faces whose ghost nodes Apollo takes
    from the last neighbour read): face 1 at order 2, face 2 at orders 3-4."""
    used = 1 if N == 2 else 2
    return int(sum(1 for c in conn if c[2 * used] < 0 and any(c[2 * j] >= 0 for j in range(used))))


def one_tag_per_element(mesh):
    """Give every boundary face of an element the tag of its first boundary
    face.  Apollo stores one boundary tag per element (the last of its
    boundary faces to be labelled writes all six connectivity slots,
    wxnodaldggeometry2d.cc:348-356), this library one per face; on meshes
    like this the two agree."""
    ft = mesh.face_tag.copy()
    for e in range(ft.shape[0]):
        tags = [t for t in ft[e] if t > 0]
        if len(set(tags)) > 1:
            ft[e][ft[e] > 0] = tags[0]
    mesh.face_tag = ft
    return mesh


# Right-hand sides made by Apollo's own code (tests/golden/make_apollo_rhs.py)
APOLLO_DIR = os.path.join(HERE, "apollo_rhs")
APOLLO_NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(APOLLO_DIR, "*.npz")))
BC_KINDS = {v: k for k, v in BC_NAMES.items()}
SRC_CODES = {"tranverseMagneticSrc": 1, "pointCurrentSrc": 2}


def load_apollo(name):
    z = np.load(os.path.join(APOLLO_DIR, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["mesh"] = Mesh(vx=d["vx"], vy=d["vy"], etov=d["etov"], face_tag=d["face_tag"], vert_canon=d["vert_canon"],
                     n=0, lo=(0, 0), hi=(1, 1), periodic=False)
    d["equation"] = str(d["equation"])
    d["numflux"] = str(d["numflux"])
    d["bcs"] = tuple((str(n), tuple(p[:k])) for n, p, k in zip(d["bc_names"], d["bc_params"], d["bc_nparams"]))
    d["sources"] = tuple((str(k), (2,), tuple(p[:n])) for k, p, n in
                         zip(d["src_kinds"], d["src_params"], d["src_nparams"]))
    return d
