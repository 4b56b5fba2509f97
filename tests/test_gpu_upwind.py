"""The upwind flux for advection (an extension: dissipation |n.u| where
Apollo's Lax-Friedrichs flux uses max(|ux|, |uy|)), on the B200 against the
oracle's restatement of the same flux: right-hand side, steps, the fused
float64 stage, mixed precision and the derivatives."""
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
