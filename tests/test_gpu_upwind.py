"""The upwind fluxes (an extension of Apollo's Lax-Friedrichs ones): for
advection, dissipation |n.u| where Apollo uses max(|ux|, |uy|); for the
planar Maxwell TM form, no dissipation on the normal magnetic field.  On the
B200 against the oracle's restatement of the same fluxes: right-hand side,
steps, the fused float64 stage, mixed precision and the derivatives."""
import os

import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import rel_l2

pytestmark = pytest.mark.gpu


def _case(orc, n=12, N=3):
    p = problems.advection(n=n, N=N)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, numerical_flux="upwind")
    o = orc.Oracle(p.mesh, p.N, orc.EQ_ADVECTION, tuple(p.eq_params)[:3] + (orc.NF_UPWIND,), cfl=p.cfl)
    o.set_threads(os.cpu_count() or 1)
    return p, s, o


def test_upwind_rhs_and_steps_match_oracle(oracle_lib):
    orc = oracle_lib
    p, s, o = _case(orc)
    rng = np.random.default_rng(1)
    U = rng.standard_normal(s.shape)
    r, sugg = s.step(0.1, 0.0, U)
    ro, so = o.rhs(U, 0.1, 0.0)
    assert rel_l2(r, ro) <= 1e-12
    assert sugg == pytest.approx(so, rel=1e-14)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    t, dt = s.advance(30, 0.0, dt0)
    Uc = U0.copy()
    n, tc, dtc = o.run(Uc, 30, 0.0, o.init_dt(U0))
    assert rel_l2(s.get_state(), Uc) <= 1e-12
    assert t == pytest.approx(tc, rel=1e-13)
    # it is not Apollo's flux: the same run with Lax-Friedrichs differs
    lf = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    lf.set_state(U0)
    lf.advance(30, 0.0, dt0)
    assert rel_l2(lf.get_state(), Uc) > 1e-6


def test_upwind_in_every_form(oracle_lib):
    orc = oracle_lib
    p, s, o = _case(orc)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    s.advance(20, 0.0, dt0)
    ref = s.get_state()
    s.set_fp64_kernels(True)
    s.set_state(U0)
    s.advance(20, 0.0, dt0)
    assert rel_l2(s.get_state(), ref) <= 1e-13
    s.set_fp64_kernels(False)
    s.set_state(U0)
    s.advance(20, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), ref) <= 1e-6
    # the right-hand side's adjoint is the transpose of its tangent
    rng = np.random.default_rng(3)
    v, w = rng.standard_normal(s.shape), rng.standard_normal(s.shape)
    jv = s.rhs_jvp(0.0, U0, v)
    jtw = s.rhs_vjp(0.0, U0, w)
    scale = np.linalg.norm(w) * np.linalg.norm(jv) + np.linalg.norm(jtw) * np.linalg.norm(v)
    assert abs(float(np.vdot(w, jv)) - float(np.vdot(jtw, v))) <= 1e-13 * scale


def test_tm_upwind_matches_oracle(oracle_lib):
    """The planar Maxwell TM form with the upwind extension (no dissipation on
    the normal magnetic field) against the oracle's restatement on the full
    field set, PEC walls: right-hand side of a random state, 20 steps of the
    cavity mode, the mixed form, and the adjoint as the tangent's transpose."""
    orc = oracle_lib
    p = problems.maxwell_tm(n=10, N=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, numerical_flux="upwind")
    o = orc.Oracle(p.mesh, p.N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0, orc.NF_UPWIND), bcs=((orc.BC_TM, ()),), cfl=p.cfl)
    o.set_threads(os.cpu_count() or 1)
    rng = np.random.default_rng(8)
    U3 = rng.uniform(-1, 1, s.shape)
    U8 = np.zeros(U3.shape[:2] + (8,))
    U8[..., 2:5] = U3
    r, sugg = s.step(0.2, 0.0, U3)
    ro, so = o.rhs(U8, 0.2, 0.0)
    assert rel_l2(r, ro[..., 2:5]) <= 1e-12
    assert sugg == pytest.approx(so, rel=1e-14)
    lf = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    assert rel_l2(lf.step(0.2, 0.0, U3)[0], r) > 1e-6  # not Apollo's flux
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    U8[...] = 0.0
    U8[..., 2:5] = U0
    s.set_state(U0)
    dt0 = s.init_dt()
    t, dt = s.advance(20, 0.0, dt0)
    U = s.get_state()
    n, tc, dtc = o.run(U8, 20, 0.0, o.init_dt(U8))
    assert rel_l2(U, U8[..., 2:5]) <= 1e-12
    assert t == pytest.approx(tc, rel=1e-13)
    s.set_state(U0)
    s.advance(20, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= 1e-6
    v, w = rng.standard_normal(s.shape), rng.standard_normal(s.shape)
    jv = s.rhs_jvp(0.0, U0, v)
    jtw = s.rhs_vjp(0.0, U0, w)
    scale = np.linalg.norm(w) * np.linalg.norm(jv) + np.linalg.norm(jtw) * np.linalg.norm(v)
    assert abs(float(np.vdot(w, jv)) - float(np.vdot(jtw, v))) <= 1e-13 * scale
