"""Generate the golden fixtures under tests/golden/ (run in the development container).

Each fixture is a small seeded case of one benchmark problem: the mesh arrays,
the initial state, one right-hand side with its suggested dt, the initial dt,
and the state after a few SSPRK(5,2) steps with Apollo's dt policy.  They are
produced by the CPU oracle with Apollo's own equation plugins compiled
unmodified (oracle/_ref/libapollo_ref.so, the per-point flux and numerical flux
hooks are the reference code); initial states are cross-checked against
Apollo's own exprFunc evaluating the example inputs' expressions.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from apollo_b200 import problems  # noqa: E402
from oracle import oracle as orc  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

VORTEX_BC = (1.0, 0.0, 5.0, 5.0, 1.4, 5.0)  # u0, v0, x0, y0, gas_gamma, beta


def gmsh_vortex(N: int = 3):
    """The Euler vortex on the unstructured Gmsh mesh square_delaunay.msh
    (make_gmsh.py), the exact vortex imposed on both boundary tags, as Apollo's
    isentropicVortex example does with isentropicVortexBC."""
    from apollo_b200.gmsh import read_gmsh
    mesh = read_gmsh(os.path.join(HERE, "square_delaunay.msh"))
    return problems.Problem("gmsh_vortex", N, 0.5, "eulerEqn", (1.4, 0.0, 0.0), mesh, (), 0,
                            ic=lambda x, y: problems.vortex_ic(x, y, 5, beta=5.0))

def channel(N: int = 3, n: int = 7, seed: int = 2):
    """Euler flow through [0,2] x [0,1] (5 fields): bottom wall (tag 1), right
    zero-gradient outflow (2), top inflow (3), left Dirichlet state (4); a
    density bump and a transverse velocity wave on a uniform stream."""
    from apollo_b200.mesh import jittered_square
    mesh = jittered_square(n, (0.0, 0.0), (2.0, 1.0), seed=seed, periodic=False, wall_tag=1)
    for f, (i, j) in enumerate(((0, 1), (1, 2), (2, 0))):
        xa, ya = mesh.vx[mesh.etov[:, i]], mesh.vy[mesh.etov[:, i]]
        xb, yb = mesh.vx[mesh.etov[:, j]], mesh.vy[mesh.etov[:, j]]
        mesh.face_tag[:, f] = np.select([(ya == 0) & (yb == 0), (xa == 2) & (xb == 2), (ya == 1) & (yb == 1),
                                         (xa == 0) & (xb == 0)], [1, 2, 3, 4], 0)

    def ic(x, y):
        rho = 1.0 + 0.2 * np.exp(-((x - 1.0) ** 2 + (y - 0.5) ** 2) / 0.05)
        u, v, p = 0.5 + 0 * x, 0.1 * np.sin(np.pi * x), 1.0 + 0 * x
        return np.stack([rho, rho * u, rho * v, 0 * x, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=-1)

    return problems.Problem("channel", N, 0.5, "eulerEqn", (1.4, 0.0, 0.0), mesh, (), 0, ic=ic)


CHANNEL_BCS = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()),
               (orc.BC_EULER_INFLOW, (0.4, -60.0, 1.4, 1.0, 1.0)),
               (orc.BC_EULER_DIRICHLET, (1.0, 0.5, 0.0, 0.0, 1.4, 1.0)))

CASES = [
    # name, builder, kwargs, oracle eq, eq params, ref kind, ref params, bcs, steps
    ("adv_N3", problems.advection, dict(n=8, N=3), orc.EQ_ADVECTION, (1.0, 0.5, 0.0), "advectionEqn",
     dict(ux=1.0, uy=0.5), (), 4),
    ("adv_N2", problems.advection, dict(n=7, N=2, seed=3), orc.EQ_ADVECTION, (1.0, 0.5, 0.0), "advectionEqn",
     dict(ux=1.0, uy=0.5), (), 4),
    ("euler_N4", problems.euler_vortex, dict(n=7, N=4, fields=5), orc.EQ_EULER, (1.4, 0.0, 0.0), "eulerEqn",
     dict(gas_gamma=1.4), (), 3),
    ("euler_N3", problems.euler_vortex, dict(n=8, N=3, fields=5, seed=5), orc.EQ_EULER, (1.4, 0.0, 0.0), "eulerEqn",
     dict(gas_gamma=1.4), (), 3),
    ("maxwell_N5", problems.maxwell_tm, dict(n=6, N=5, fields=8), orc.EQ_MAXWELL, (1.0, 0.0, 0.0), "phMaxwellEqn",
     dict(c0=1.0), ((orc.BC_TM, ()),), 3),
    ("maxwell_N2", problems.maxwell_tm, dict(n=7, N=2, fields=8, seed=2), orc.EQ_MAXWELL, (1.0, 0.0, 0.0),
     "phMaxwellEqn", dict(c0=1.0), ((orc.BC_TM, ()),), 3),
    ("euler_gmsh_N3", gmsh_vortex, dict(N=3), orc.EQ_EULER, (1.4, 0.0, 0.0), "eulerEqn", dict(gas_gamma=1.4),
     ((orc.BC_VORTEX, VORTEX_BC), (orc.BC_VORTEX, VORTEX_BC)), 3),
    ("euler_hll_N3", channel, dict(N=3), orc.EQ_EULER, (1.4, 0.0, 0.0, orc.NF_HLL), "eulerEqn",
     dict(gas_gamma=1.4, Numerical_Flux="HLL"), CHANNEL_BCS, 3),
    ("euler_roe_N4", channel, dict(N=4, seed=3), orc.EQ_EULER, (1.4, 0.0, 0.0, orc.NF_ROE), "eulerEqn",
     dict(gas_gamma=1.4, Numerical_Flux="Roe"), CHANNEL_BCS, 0),  # Apollo's Roe flux is non-physical within a step
    ("euler_wave_N2", channel, dict(N=2, n=8), orc.EQ_EULER, (1.4, 0.0, 0.0, orc.NF_WAVE), "eulerEqn",
     dict(gas_gamma=1.4, Numerical_Flux="Wave"), CHANNEL_BCS, 1),  # non-physical from the second step
    ("euler_hll_limiter_N3", channel, dict(N=3, n=9, seed=4), orc.EQ_EULER, (1.4, 0.0, 0.0, orc.NF_HLL), "eulerEqn",
     dict(gas_gamma=1.4, Numerical_Flux="HLL"), CHANNEL_BCS, 4),
    ("euler_hll_talimiter_N3", channel, dict(N=3, n=9, seed=6), orc.EQ_EULER, (1.4, 1e-6, 1e-6, orc.NF_HLL),
     "eulerEqn", dict(gas_gamma=1.4, Numerical_Flux="HLL", minPressure=1e-6, minDensity=1e-6), CHANNEL_BCS, 4),
    ("maxwell_talimiter_N3", problems.maxwell_tm, dict(n=6, N=3, fields=8, seed=7), orc.EQ_MAXWELL, (1.0, 0.0, 0.0),
     "phMaxwellEqn", dict(c0=1.0), ((orc.BC_TM, ()),), 3),
    ("maxwell_src_N3", problems.maxwell_tm, dict(n=7, N=3, fields=8, seed=8), orc.EQ_MAXWELL, (1.0, 1.0, 1.0),
     "phMaxwellEqn", dict(c0=1.0, gamma=1.0, chi=1.0), ((orc.BC_PEC, ()),), 4),
]

# source plugins per case (kind, Apollo output field, params), Apollo's example
# TM2DwithSource.pin (tranverseMagneticSrc into Ez, phMaxwellEqn with chi =
# gamma = 1, conducting walls) plus a point current into Ez
SOURCES = {"maxwell_src_N3": ((orc.SRC_TM, 2, ()),
                              (orc.SRC_POINT, 2, (0.4, 0.6, 0.15, 2.0, 5.0, 0.2, 1.0, 1.0, 1.0)))}
SRC_NAMES = {orc.SRC_TM: "tranverseMagneticSrc", orc.SRC_POINT: "pointCurrentSrc"}

# the limiter per case: eulerLimiterHW with its own (gas_gamma, min_pressure,
# min_density), or tuAliabadiLimiter, which takes the equation's parameters
LIMITERS = {"euler_hll_limiter_N3": ("eulerLimiterHW", (1.4, 1e-6, 1e-6)),
            "euler_hll_talimiter_N3": ("tuAliabadiLimiter", ()),
            "maxwell_talimiter_N3": ("tuAliabadiLimiter", ())}

FLUX_NAMES = {orc.NF_LF: "LF", orc.NF_HLL: "HLL", orc.NF_ROE: "Roe", orc.NF_WAVE: "Wave"}


def make_case(name, builder, kw, eq, eqp, ref_kind, ref_params, bcs, steps, ref):
    prob = builder(**kw)
    mesh = prob.mesh
    o = orc.Oracle(mesh, prob.N, eq, eqp, bcs=bcs, cfl=prob.cfl)
    eh = ref.equation(ref_kind, **ref_params)
    o.use_ref_plugins(ref, eh)
    x, y = o.node_coords()
    U0 = np.ascontiguousarray(prob.ic(x, y), dtype=np.float64)
    lim = LIMITERS.get(name)
    extra = {}
    srcs = SOURCES.get(name, ())
    for kind, out, params in srcs:
        o.add_source(kind, out, params)
    if srcs:
        extra["src_kinds"] = np.asarray([SRC_NAMES[k] for k, _, _ in srcs])
        extra["src_out"] = np.asarray([out for _, out, _ in srcs], dtype=np.int32)
        extra["src_params"] = np.asarray([list(p) + [0.0] * (9 - len(p)) for _, _, p in srcs], dtype=np.float64)
        extra["src_nparams"] = np.asarray([len(p) for _, _, p in srcs], dtype=np.int32)
    if lim is not None:
        # the limiter (restated in the oracle; Apollo's needs PETSc's DMPlex)
        # acts on every stage input, and on the input of a single right-hand side
        kind, params = lim
        if kind == "eulerLimiterHW":
            o.set_limiter(*params)
        else:
            o.set_limiter_ta()
        extra["limiter"] = np.asarray(params, dtype=np.float64)
        extra["limiter_kind"] = kind
        rhs, sugg = o.rhs(o.limit(U0), 0.0, 0.0)
    else:
        rhs, sugg = o.rhs(U0, 0.0, 0.0)
    dt0 = o.init_dt(U0)
    U = U0.copy()
    n, t, dt = o.run(U, steps, 0.0, dt0)
    assert n == steps and o.error == 0
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        vx=mesh.vx, vy=mesh.vy, etov=mesh.etov, face_tag=mesh.face_tag, vert_canon=mesh.vert_canon,
        N=prob.N, cfl=prob.cfl, eq=eq, eqp=np.asarray(list(eqp) + [0.0] * (4 - len(eqp)), dtype=np.float64),
        equation=ref_kind, numflux=FLUX_NAMES[int(eqp[3]) if len(eqp) > 3 else 0],
        bc_kinds=np.asarray([b[0] for b in bcs], dtype=np.int32),
        bc_params=np.asarray([list(b[1]) + [0.0] * (8 - len(b[1])) for b in bcs], dtype=np.float64).reshape(-1, 8),
        x=x, y=y, U0=U0, rhs=rhs, sugg=sugg, dt0=dt0,
        steps=steps, U_end=U, t_end=t, dt_end=dt, **extra)
    return name, U0.shape, float(np.abs(rhs).max())


def main(names=()):
    """All cases, or only those named on the command line."""
    orc.build(with_ref=True)
    ref = orc.RefPlugins()
    for case in CASES:
        if not names or case[0] in names:
            print(make_case(*case, ref=ref))


if __name__ == "__main__":
    main(sys.argv[1:])
