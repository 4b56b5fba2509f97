"""The fused mixed-precision stage kernel (four-field Euler, Lax-Friedrichs,
orders 2..4) against the float64 path and against the chunked mixed kernel
(B200).

The fused kernel holds the whole tile's flux-deviation operand in shared
memory and writes the result's face traces with a tensor-core interpolation;
its arithmetic is the chunked kernel's deviation form, so both stay within the
mixed form's error of float64 and of each other.
"""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from apollo_b200.mesh import jittered_square
from golden_cases import rel_l2

pytestmark = pytest.mark.gpu

VB = (1.0, 0.3, 1.0, 0.5, 1.4, 2.0)  # isentropicVortexBC: u0, v0, x0, y0, gamma, beta


def _walls(N, n=9):
    """A non-periodic jittered mesh with the vortex condition on every side and
    a random physical state: boundary faces and all three face kinds."""
    mesh = jittered_square(n, (0.0, 0.0), (2.0, 1.0), seed=N, periodic=False)
    s = NodalDG2d(N, 0.5, "eulerEqn2d", (1.4, 0.0, 0.0), mesh, bcs=(("isentropicVortexBC", VB),))
    rng = np.random.default_rng(7 + N)
    U = 0.1 * rng.uniform(-1, 1, (mesh.K, s.Np, 4))
    U[..., 0] += 1.0
    U[..., 1] += 0.5
    U[..., 3] = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2) / U[..., 0] + 2.0 + U[..., 3]
    return s, np.ascontiguousarray(U)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_fused_rhs_with_boundaries(N):
    s, U = _walls(N)
    r64, s64 = s.step(0.3, 0.01, U)
    s.set_launch_shape(1, 0)
    rf, sf = s.step(0.3, 0.01, U, precision="mixed")
    s.set_launch_shape(1, 2)
    rc, sc = s.step(0.3, 0.01, U, precision="mixed")
    # the forward-Euler stage with the stepper's dt
    s.set_state(U)
    dt = s.init_dt()
    e_f = rel_l2(U + dt * rf, U + dt * r64)
    e_c = rel_l2(U + dt * rc, U + dt * r64)
    print(N, "stage fused", e_f, "chunked", e_c, "rhs fused", rel_l2(rf, r64))
    assert e_f <= 1e-6
    assert rel_l2(rf, r64) <= 1e-4
    assert rel_l2(rf, rc) <= 1e-5
    assert sf == pytest.approx(s64, rel=1e-6)
    assert sf == pytest.approx(sc, rel=1e-6)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_fused_steps_with_boundaries(N):
    s, U = _walls(N)
    s.set_state(U)
    dt = s.init_dt()
    t64, d64 = s.advance(4, 0.3, dt)
    U64 = s.get_state()
    s.set_launch_shape(1, 0)
    s.set_state(U)
    tf, df = s.advance(4, 0.3, dt, precision="mixed")
    e = rel_l2(s.get_state(), U64)
    print(N, "4 steps fused vs float64", e)
    assert e <= 1e-6
    assert tf == pytest.approx(t64, rel=1e-7)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_fused_vortex_steps(N):
    """Periodic vortex, 40 steps: fused vs float64 and vs the chunked kernel,
    and every grid share giving the same result."""
    p = problems.euler_vortex(n=33, N=N)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    s.advance(40, 0.0, dt0)
    U64 = s.get_state()
    ends = {}
    for share, shape in ((1, 0), (3, 0), (1, 2)):
        s.set_launch_shape(share, shape)
        s.set_state(U0)
        s.advance(40, 0.0, dt0, precision="mixed")
        ends[(share, shape)] = s.get_state()
    np.testing.assert_array_equal(ends[(1, 0)], ends[(3, 0)])
    e_f, e_c = rel_l2(ends[(1, 0)], U64), rel_l2(ends[(1, 2)], U64)
    print(N, "40 steps fused", e_f, "chunked", e_c)
    assert e_f <= 1e-6
    assert rel_l2(ends[(1, 0)], ends[(1, 2)]) <= 5e-7


def test_fused_ragged_last_tile():
    """K not a multiple of the 32-element tile (and fewer tiles than SMs)."""
    mesh = jittered_square(6, (0.0, 0.0), (1.0, 1.0), seed=3, periodic=True)  # K = 50
    s = NodalDG2d(4, 0.5, "eulerEqn2d", (1.4, 0.0, 0.0), mesh)
    x, y = s.node_coords()
    from apollo_b200.problems import vortex_ic
    U0 = np.ascontiguousarray(vortex_ic(5 * x + 2.5, 5 * y + 2.5, 4))
    r64, _ = s.step(0.0, 0.0, U0)
    rf, _ = s.step(0.0, 0.0, U0, precision="mixed")
    s.set_state(U0)
    dt = s.init_dt()
    assert rel_l2(U0 + dt * rf, U0 + dt * r64) <= 1e-6
    s.advance(3, 0.0, dt)
    U64 = s.get_state()
    s.set_state(U0)
    s.advance(3, 0.0, dt, precision="mixed")
    assert rel_l2(s.get_state(), U64) <= 1e-6
