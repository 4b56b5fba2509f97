"""Golden right-hand sides made by Apollo's own code.

Each fixture holds a mesh, a state and the right-hand side and suggested dt
that Apollo's WxNodalDG2dMethod computes for it (with a limiter in its
Limiter list where the fixture names one), and for some a few SSPRK(5,2)
steps taken through it, run compiled unmodified
through oracle/ref_driver.cpp (`make -C oracle refdrv`, which needs Apollo's
source tree).  The B200 tests compare the CUDA path with these directly.
Run from the repository root: python tests/golden/make_apollo_rhs.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from apollo_b200.mesh import jittered_square  # noqa: E402
from golden_cases import (CHANNEL_DIRICHLET, CHANNEL_INFLOW, channel_mesh, channel_state,  # noqa: E402
                          one_tag_per_element)
from oracle import oracle as orc  # noqa: E402

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "apollo_rhs")
EULER_BCS = (("eulerWallBC", ()), ("eulerZeroGradientBC", ()), ("eulerInflowBC", CHANNEL_INFLOW),
             ("eulerDirichletBC", CHANNEL_DIRICHLET))
BC_KEYS = {"eulerInflowBC": ("Mach_number", "Flow_angle", "gas_gamma", "Pressure", "density"),
           "eulerDirichletBC": ("density", "xvelocity", "yvelocity", "zvelocity", "gas_gamma", "pressure"),
           "isentropicVortexBC": ("u0", "v0", "x0", "y0", "gas_gamma", "beta"),
           "gridFixedBC": ("value",)}
SRC_KEYS = ("xLocation", "yLocation", "radius", "currentDensity", "frequency", "phase", "charge", "mass", "epsilon0")
VORTEX = ["r = sqrt((x-xo)*(x-xo)+(y-yo)*(y-yo))", "u = uo - beta*exp(1.-r*r)*(y-yo)/(2.*pi)",
          "v = vo + beta*exp(1.-r*r)*(x-xo)/(2.*pi)",
          "base = 1. - ( (gamma-1.)*beta*beta*exp(2.*(1.-r*r))/(16.*gamma*pi*pi) )", "rho = base^(1./(gamma-1.))",
          "p   = rho^gamma", "en = p/(gamma-1.) + 0.5*rho*(u*u + v*v)", "rhou = rho*u", "rhov = rho*v"]
FIELDS = {"eulerEqn": 5, "phMaxwellEqn": 8, "advectionEqn": 1}


def deck(N, eq, bcs, meqn, exprs=None, keys="", consts="", progn=None, blocks=""):
    exprs = exprs or ["0.0"] * meqn
    pg = "" if progn is None else "  progn = [" + ", ".join(f'"{p}"' for p in progn) + "]\n"
    return (f"<hyperbolic>\n Kind = nodalDG2d\n Equations = [eq]\n boundaryConditions = [{', '.join(bcs)}]\n"
            f" polynomialOrder = {N}\n cfl = 0.5\n DataStructure = [0, dg, {meqn * (N + 1) * (N + 2) // 2}]\n{keys}"
            f" <InitialCondition>\n  Kind = exprFunc\n{consts}  exprList = [" + ", ".join(f'"{e}"' for e in exprs)
            + f"]\n{pg} </InitialCondition>\n{blocks} <eq>\n{eq}\n </eq>\n</hyperbolic>\n")


def save(name, mesh, N, equation, eqp, flux, bcs, U, t, dt, r, sources=(), steps=0, limiter=None):
    """The right-hand side at (U, t, dt) and, with `steps`, that many
    SSPRK(5,2) steps from (U, t = 0, dt) through the same code."""
    rhs, sugg = r.rhs(U, t, dt)
    extra = {}
    if steps:
        U_end, t_end, dt_end = r.run(U, steps, 0.0, dt)
        extra = dict(steps=steps, U_end=U_end, t_end=t_end, dt_end=dt_end)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), vx=mesh.vx, vy=mesh.vy, etov=mesh.etov, face_tag=mesh.face_tag,
        vert_canon=mesh.vert_canon, N=N, equation=equation, eqp=np.asarray(eqp, dtype=np.float64), numflux=flux,
        bc_names=np.asarray([b[0] for b in bcs]),
        bc_params=np.asarray([list(b[1]) + [0.0] * (8 - len(b[1])) for b in bcs], dtype=np.float64).reshape(-1, 8),
        bc_nparams=np.asarray([len(b[1]) for b in bcs], dtype=np.int32),
        src_kinds=np.asarray([s[0] for s in sources]), src_params=np.asarray(
            [list(s[1]) + [0.0] * (9 - len(s[1])) for s in sources], dtype=np.float64).reshape(-1, 9),
        src_nparams=np.asarray([len(s[1]) for s in sources], dtype=np.int32),
        U=U, t=t, dt=dt, rhs=rhs, sugg=sugg, **extra,
        **({} if limiter is None else dict(limiter_kind=limiter[0],
                                           limiter=np.asarray(limiter[1], dtype=np.float64))))
    print(name, U.shape, float(np.abs(rhs).max()))


def driver(mesh, bcs):
    r = orc.RefDriver(mesh)
    for i, (kind, params) in enumerate(bcs):
        r.add_bc(f"bc{i + 1}", kind, **dict(zip(BC_KEYS.get(kind, ()), params)))
    return r, [f"bc{i + 1}" for i in range(len(bcs))]


def main():
    os.makedirs(HERE, exist_ok=True)
    orc.build(with_ref=True)
    cases = [("LF", N) for N in (2, 3, 4, 5)] + [(f, N) for f in ("HLL", "Roe", "Wave") for N in (3, 4)]
    for flux, N in cases:
        mesh = one_tag_per_element(channel_mesh(5, seed=N, rotate_seed=N))
        r, names = driver(mesh, EULER_BCS)
        r.setup(deck(N, f"  Kind = eulerEqn\n  gas_gamma = 1.4\n  Numerical_Flux = {flux}", names, 5))
        o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0))
        x, y = o.node_coords()
        U = channel_state(x, y, rough=0.05, seed=N)
        _, dt0 = r.rhs(U, 0.0, 0.0)  # Apollo's suggested dt at this state
        # steps only with LF and HLL: Apollo's Roe and Wave fluxes turn the
        # state non-physical within a step or two, where Apollo's driver exits
        save(f"euler_{flux.lower()}_channel_N{N}", mesh, N, "eulerEqn", (1.4, 0.0, 0.0), flux, EULER_BCS,
             U, 0.3, dt0, r, steps=3 if flux in ("LF", "HLL") else 0)
    # each limiter in the method's Limiter list (the limiter acts on every
    # stage input), HLL flux, the channel's four conditions
    for kind, N in (("eulerLimiterHW", 3), ("tuAliabadiLimiter", 4)):
        mesh = one_tag_per_element(channel_mesh(5, seed=N + 20, rotate_seed=N + 20))
        r, names = driver(mesh, EULER_BCS)
        eq = "  Kind = eulerEqn\n  gas_gamma = 1.4\n  Numerical_Flux = HLL"
        if kind == "eulerLimiterHW":
            r.add_limiter("lim", kind, names, gas_gamma=1.4, min_pressure=1e-6, min_density=1e-6)
            eqp, lim = (1.4, 0.0, 0.0), (kind, (1.4, 1e-6, 1e-6))
        else:
            r.add_limiter("lim", kind, names, equation="eulerEqn", gas_gamma=1.4, minPressure=1e-6,
                          minDensity=1e-6)
            eq += "\n  minPressure = 1e-6\n  minDensity = 1e-6"
            eqp, lim = (1.4, 1e-6, 1e-6), (kind, ())
        r.setup(deck(N, eq, names, 5, keys=" Limiter = [lim]\n"))
        o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0))
        x, y = o.node_coords()
        U = channel_state(x, y, rough=0.15, seed=N)
        _, dt0 = r.rhs(U, 0.0, 0.0)
        save(f"euler_hll_{'hw' if kind == 'eulerLimiterHW' else 'ta'}limiter_channel_N{N}", mesh, N, "eulerEqn",
             eqp, "HLL", EULER_BCS, U, 0.3, dt0, r, steps=3, limiter=lim)
    # Apollo's isentropicVortex example on a walled square
    N = 4
    mesh = jittered_square(7, (0.0, -5.0), (10.0, 5.0), seed=N, periodic=False, wall_tag=1)
    bcs = (("isentropicVortexBC", (1.0, 0.0, 5.0, 0.0, 1.4, 5.0)),)
    r, names = driver(mesh, bcs)
    consts = "".join(f"  {k} = {v}\n" for k, v in (("xo", 5.0), ("yo", 0.0), ("beta", 5.0), ("gamma", 1.4),
                                                    ("uo", 1.0), ("vo", 0.0), ("pi", 3.141592653589793)))
    r.setup(deck(N, "  Kind = eulerEqn\n  gas_gamma = 1.4", names, 5, ["rho", "rhou", "rhov", "0.0", "en"],
                 consts=consts, progn=VORTEX))
    u0, dt0 = r.init(0.0)
    save("euler_vortex_N4", mesh, N, "eulerEqn", (1.4, 0.0, 0.0), "LF", bcs, u0, 0.3, dt0, r, steps=5)
    rng = np.random.default_rng(11)
    # Maxwell TM cavity, order 5
    N = 5
    mesh = jittered_square(5, seed=N, periodic=False, wall_tag=1)
    bcs = (("maxwellTransverseMagneticBC", ()),)
    r, names = driver(mesh, bcs)
    r.setup(deck(N, "  Kind = phMaxwellEqn\n  c0 = 1.0", names, 8))
    Np = (N + 1) * (N + 2) // 2
    U = rng.standard_normal((mesh.K, Np, 8))
    save("maxwell_tm_N5", mesh, N, "phMaxwellEqn", (1.0, 0.0, 0.0), "LF", bcs, U, 0.3, r.rhs(U, 0.0, 0.0)[1], r,
         steps=3)
    # cleaned Maxwell, conducting walls, TM2DwithSource.pin's source and a point current
    N = 3
    mesh = jittered_square(5, seed=N, periodic=False, wall_tag=1)
    bcs = (("phmConductingWallBC", ()),)
    pc = (0.4, 0.6, 0.15, 2.0, 5.0, 0.2, 1.0, 2.0, 0.5)
    r, names = driver(mesh, bcs)
    blocks = (" <current>\n  Kind = tranverseMagneticSrc\n  OutRange = [2]\n </current>\n <wire>\n"
              "  Kind = pointCurrentSrc\n  OutRange = [2]\n" + "".join(f"  {k} = {v}\n" for k, v in zip(SRC_KEYS, pc))
              + " </wire>\n")
    r.setup(deck(N, "  Kind = phMaxwellEqn\n  c0 = 1.0\n  chi = 1.0\n  gamma = 1.0", names, 8,
                 keys=" Sources = [current, wire]\n", blocks=blocks))
    Np = (N + 1) * (N + 2) // 2
    U = rng.standard_normal((mesh.K, Np, 8))
    save("maxwell_src_N3", mesh, N, "phMaxwellEqn", (1.0, 1.0, 1.0), "LF", bcs, U, 0.7, r.rhs(U, 0.0, 0.0)[1], r,
         sources=(("tranverseMagneticSrc", ()), ("pointCurrentSrc", pc)), steps=3)
    # advection with a fixed inflow value
    mesh = jittered_square(6, seed=13, periodic=False, wall_tag=1)
    bcs = (("gridFixedBC", (0.75,)),)
    r, names = driver(mesh, bcs)
    r.setup(deck(N, "  Kind = advectionEqn\n  ux = 1.0\n  uy = 0.5", names, 1))
    U = rng.standard_normal((mesh.K, Np, 1))
    save("advection_N3", mesh, N, "advectionEqn", (1.0, 0.5, 0.0), "LF", bcs, U, 0.3, r.rhs(U, 0.0, 0.0)[1], r,
         steps=3)


if __name__ == "__main__":
    main()
