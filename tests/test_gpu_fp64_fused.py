"""The fused float64 stage kernel (B200) against the volume, face and LIFT
kernels: both evaluate Apollo's right-hand side (the fused one with every
element computing its own faces, as Apollo does), so they agree within
float64 round-off on every fixture, over whole steps, and on the periodic
vortex at the benchmark's order; the fused kernel is the one that runs."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import NAMES, load, rel_l2

pytestmark = pytest.mark.gpu


def _solver(g):
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                  numerical_flux=g["numflux"], sources=g["sources"])
    if "limiter" in g:
        s.set_limiter(str(g.get("limiter_kind", "eulerLimiterHW")), g["limiter"])
    return s


@pytest.mark.parametrize("name", NAMES)
def test_fused_matches_three_kernels(name):
    g = load(name)
    s = _solver(g)
    U0 = np.ascontiguousarray(g["U0"])
    out = {}
    for fused in (True, False):
        s.set_fp64_kernels(fused)
        r, sugg = s.step(0.0, 0.0, U0)
        s.set_state(U0)
        t, dt = s.advance(int(g["steps"]), 0.0, float(g["dt0"]))
        out[fused] = (r, sugg, s.get_state(), t, dt)
    (r1, s1, u1, t1, d1), (r0, s0, u0, t0, d0) = out[True], out[False]
    tol = 1e-11 if name.startswith("euler") else 1e-13  # the vortex RHS cancels O(1) terms
    assert rel_l2(r1, r0) <= tol
    assert s1 == pytest.approx(s0, rel=1e-14)
    assert rel_l2(u1, u0) <= 1e-13
    assert rel_l2(u1, g["U_end"]) <= 1e-12
    assert t1 == pytest.approx(t0, rel=1e-15) and d1 == pytest.approx(d0, rel=1e-14)


@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_fused_vortex_steps(N):
    p = problems.euler_vortex(n=20, N=N)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    ends = {}
    for fused in (True, False):
        s.set_fp64_kernels(fused)
        s.set_state(U0)
        s.advance(10, 0.0, s.init_dt())
        ends[fused] = s.get_state()
    assert rel_l2(ends[True], ends[False]) <= 1e-13
    # conservation over the periodic square holds to round-off in the fused form
    s.set_fp64_kernels(True)
    s.set_state(U0)
    m0 = s.integrals()
    s.advance(10, 0.0, s.init_dt())
    m1 = s.integrals()
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(m0).max())


def test_auto_form_picks_by_mesh_size():
    """Form 2: the fused kernel on a mesh of one wave of tiles (one launch per
    stage), the three kernels on the benchmark mesh."""
    for n, fused_expected in ((24, True), (256, False)):
        p = problems.euler_vortex(n=n, N=4)
        s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
        x, y = s.node_coords()
        s.set_state(np.ascontiguousarray(p.ic(x, y)))
        s.set_fp64_kernels(2)
        kt = s.kernel_times(2)
        assert (kt[1] < 0.2 * kt[0] and kt[2] < 0.2 * kt[0]) == fused_expected
        s.close()


def test_fused_kernel_is_the_one_that_runs():
    p = problems.euler_vortex(n=24, N=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    s.set_state(np.ascontiguousarray(p.ic(x, y)))
    s.set_fp64_kernels(True)
    kt = s.kernel_times(3)
    assert kt[0] > 0 and kt[1] < 0.2 * kt[0] and kt[2] < 0.2 * kt[0]  # one kernel: no face or LIFT launch
    s.set_fp64_kernels(False)
    kt3 = s.kernel_times(3)
    assert kt3[1] > 0 and kt3[2] > 0
