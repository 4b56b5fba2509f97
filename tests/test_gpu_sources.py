"""Source plugins on the device (B200): Apollo's tranverseMagneticSrc and
pointCurrentSrc evaluated at the cubature points at the stage time and added
to the volume term as V^T (w J S), against the oracle (which evaluates them as
Apollo's source set does, pinned bit for bit to the compiled plugins) in every
form: float64, the planar Maxwell TM form, mixed precision (the chunked and
the fused stage kernels), the no-allocation right-hand side."""
import ctypes as C
import os

import numpy as np
import pytest

from apollo_b200 import ApolloError, NodalDG2d, problems
from apollo_b200.mesh import jittered_square
from golden_cases import load, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
WIRE = (0.4, 0.6, 0.15, 2.0, 5.0, 0.2, 1.0, 1.0, 1.0)


def test_planar_tm_with_sources_equals_full_maxwell():
    """maxwellTM (Ez, Bx, By) with the sources into Ez equals phMaxwellEqn's
    fixture (chi = gamma = 1 there, so only the TM triple is compared after
    one right-hand side of a state whose other fields are zero)."""
    g = load("maxwell_src_N3")
    mesh = g["mesh"]
    srcs = (("tranverseMagneticSrc", (2,), ()), ("pointCurrentSrc", (2,), WIRE))
    s8 = NodalDG2d(3, 0.5, "phMaxwellEqn", (1.0, 0.0, 0.0), mesh, bcs=(("maxwellTransverseMagneticBC", ()),),
                   sources=srcs)
    s3 = NodalDG2d(3, 0.5, "maxwellTM", (1.0,), mesh, bcs=(("maxwellTransverseMagneticBC", ()),), sources=srcs)
    U8 = np.zeros(g["U0"].shape)
    U8[..., 2:5] = g["U0"][..., 2:5]
    r8, a8 = s8.step(0.7, 0.01, U8)
    r3, a3 = s3.step(0.7, 0.01, np.ascontiguousarray(U8[..., 2:5]))
    assert rel_l2(r3, r8[..., 2:5]) <= 1e-14
    assert a3 == a8


def test_tm_steps_match_oracle_and_mixed(oracle_lib):
    """The TM cavity with both sources, N = 4, 20 steps: float64 vs the oracle,
    mixed vs float64."""
    orc = oracle_lib
    p = problems.maxwell_tm(n=12, N=4)
    srcs = (("tranverseMagneticSrc", (2,), ()), ("pointCurrentSrc", (2,), WIRE))
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, sources=srcs)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),), cfl=p.cfl)
    o.add_source(orc.SRC_TM, 2)
    o.add_source(orc.SRC_POINT, 2, WIRE)
    o.set_threads(os.cpu_count() or 1)
    x, y = s.node_coords()
    U3 = np.ascontiguousarray(p.ic(x, y))
    U8 = np.zeros(U3.shape[:2] + (8,))
    U8[..., 2:5] = U3
    s.set_state(U3)
    dt0 = s.init_dt()
    t, dt = s.advance(20, 0.0, dt0)
    U = s.get_state()
    n, tc, dtc = o.run(U8, 20, 0.0, o.init_dt(U8))
    assert rel_l2(U, U8[..., 2:5]) <= TOL
    assert t == pytest.approx(tc, rel=1e-13)
    s.set_state(U3)
    s.advance(20, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= 1e-6
    # without the sources the run differs: they are really applied
    s0 = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    s0.set_state(U3)
    s0.advance(20, 0.0, dt0)
    assert rel_l2(s0.get_state(), U) > 1e-4


def test_source_in_fused_euler_stage(oracle_lib):
    """A point source into the energy of the Euler vortex (eulerEqn2d, the fused
    mixed kernel at N = 3): float64 vs the oracle (eulerEqn, field 4), fused
    mixed vs float64, fused vs chunked."""
    orc = oracle_lib
    p = problems.euler_vortex(n=17, N=3, fields=4)
    wire = (5.0, 5.0, 1.5, 0.5, 2.0, 0.1, 1.0, 1.0, 1.0)
    srcs = (("pointCurrentSrc", (4,), wire),)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, sources=srcs)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_EULER, p.eq_params, cfl=p.cfl)
    o.add_source(orc.SRC_POINT, 4, wire)
    x, y = s.node_coords()
    U4 = np.ascontiguousarray(p.ic(x, y))
    U5 = np.zeros(U4.shape[:2] + (5,))
    U5[..., [0, 1, 2, 4]] = U4
    r64, _ = s.step(0.3, 0.0, U4)
    ro, _ = o.rhs(U5, 0.3, 0.0)
    assert rel_l2(r64, ro[..., [0, 1, 2, 4]]) <= 1e-11  # the vortex right-hand side cancels (see parity tests)
    s.set_state(U4)
    dt0 = s.init_dt()
    s.advance(6, 0.0, dt0)
    U64 = s.get_state()
    ends = {}
    for shape in (0, 2):
        s.set_launch_shape(1, shape)
        s.set_state(U4)
        s.advance(6, 0.0, dt0, precision="mixed")
        ends[shape] = s.get_state()
    assert rel_l2(ends[0], U64) <= 1e-6
    assert rel_l2(ends[2], U64) <= 1e-6


def test_noalloc_with_sources():
    torch = pytest.importorskip("torch")
    g = load("maxwell_src_N3")
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                  sources=g["sources"])
    u = torch.from_numpy(g["U0"]).cuda()
    ref = torch.empty_like(u)
    s.step(0.25, 1e-3, u, ref)
    out = torch.empty_like(u)
    rc = s.lib.apollo_dg_rhs_noalloc(s.h, 0.25, 1e-3, C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()), None,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_source_errors():
    p = problems.maxwell_tm(n=6, N=3)
    with pytest.raises(ApolloError):  # Ex is not a field of the planar TM form
        NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, sources=(("tranverseMagneticSrc", (0,), ()),))
    with pytest.raises(ApolloError):
        NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, sources=(("noSuchSrc", (2,), ()),))
    with pytest.raises(ApolloError):  # pointCurrentSrc takes nine parameters
        NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, sources=(("pointCurrentSrc", (2,), (1.0,)),))
