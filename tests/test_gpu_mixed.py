"""Mixed-precision (tcgen05, split tf32, deviation form) path vs the float64 path (B200)."""
import numpy as np
import pytest

from apollo_b200 import ApolloError, NodalDG2d, problems
from golden_cases import LF_NAMES as NAMES, load, rel_l2

pytestmark = pytest.mark.gpu


def _solver(g):
    return NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                     numerical_flux=g["numflux"], sources=g["sources"])


@pytest.mark.parametrize("name", NAMES)
def test_mixed_rhs_close_to_fp64(name):
    g = load(name)
    s = _solver(g)
    r64, s64 = s.step(0.0, 0.0, g["U0"])
    rmx, smx = s.step(0.0, 0.0, g["U0"], precision="mixed")
    dt0 = float(g["dt0"])
    # the stage update the stepper forms, and the RHS itself.  These fixtures
    # are coarse (5-8 vertices a side), where an element's fluctuation is as
    # large as its mean and the deviation form gains little; tf32 x3 products
    # with fp32 flux leave ~1e-6 of the RHS scale.
    e_stage = rel_l2(g["U0"] + dt0 * rmx, g["U0"] + dt0 * r64)
    e_rhs = rel_l2(rmx, r64)
    print(name, "stage", e_stage, "rhs", e_rhs)
    assert e_stage <= 1e-6
    assert e_rhs <= 1e-4
    assert smx == pytest.approx(s64, rel=1e-6)


@pytest.mark.parametrize("name", NAMES)
def test_mixed_steps_close_to_fp64(name):
    g = load(name)
    s = _solver(g)
    s.set_state(g["U0"])
    dt0 = s.init_dt()
    t64, d64 = s.advance(int(g["steps"]), 0.0, dt0)
    U64 = s.get_state()
    s.set_state(g["U0"])
    tmx, dmx = s.advance(int(g["steps"]), 0.0, dt0, precision="mixed")
    Umx = s.get_state()
    e = rel_l2(Umx, U64)
    print(name, "steps", e)
    assert e <= 1e-6
    assert tmx == pytest.approx(t64, rel=1e-7)


@pytest.mark.parametrize("name", ["euler_hll_N3", "euler_roe_N4", "euler_wave_N2"])
def test_mixed_other_euler_fluxes_close_to_fp64(name):
    """HLL, Roe and Wave (Apollo's arithmetic, quirks included) in the mixed
    stage: its fp32 face flux is the equation's own, and the float64 face
    constants are that flux at the element mean, so the mixed right-hand side
    and steps track the float64 ones as closely as with Lax-Friedrichs."""
    g = load(name)
    s = _solver(g)
    r64, s64 = s.step(0.0, 0.0, g["U0"])
    rmx, smx = s.step(0.0, 0.0, g["U0"], precision="mixed")
    dt0 = float(g["dt0"])
    e_stage = rel_l2(g["U0"] + dt0 * rmx, g["U0"] + dt0 * r64)
    print(name, "stage", e_stage, "rhs", rel_l2(rmx, r64))
    assert e_stage <= 1e-6
    assert smx == pytest.approx(s64, rel=1e-5)
    if int(g["steps"]) > 0:
        s.set_state(g["U0"])
        s.advance(int(g["steps"]), 0.0, dt0)
        U64 = s.get_state()
        s.set_state(g["U0"])
        s.advance(int(g["steps"]), 0.0, dt0, precision="mixed")
        e = rel_l2(s.get_state(), U64)
        print(name, "steps", e)
        assert e <= 1e-6


@pytest.mark.parametrize("name", ["euler_hll_limiter_N3", "euler_hll_talimiter_N3", "maxwell_talimiter_N3"])
def test_mixed_with_limiter_close_to_fp64(name):
    """With a limiter the mixed stepper limits each stage input in float64 and
    rebuilds that state's face traces before the stage; a right-hand side
    limits a copy of its input.  Both track the float64 path."""
    g = load(name)
    s = _solver(g)
    r64, _ = s.step(0.0, 0.0, g["U0"])
    rmx, _ = s.step(0.0, 0.0, g["U0"], precision="mixed")
    dt0 = float(g["dt0"])
    e_stage = rel_l2(g["U0"] + dt0 * rmx, g["U0"] + dt0 * r64)
    s.set_state(g["U0"])
    s.advance(int(g["steps"]), 0.0, dt0)
    U64 = s.get_state()
    s.set_state(g["U0"])
    s.advance(int(g["steps"]), 0.0, dt0, precision="mixed")
    e = rel_l2(s.get_state(), U64)
    print(name, "stage", e_stage, "steps", e)
    assert e_stage <= 1e-6
    assert e <= 1e-6


def test_mixed_vortex_l2_after_steps():
    """Euler vortex (N = 4) on a 64 x 64 grid: mixed stays within 1e-6 relative L2 of float64."""
    p = problems.euler_vortex(n=64, N=4, fields=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    s.advance(100, 0.0, dt0)
    U64 = s.get_state()
    s.set_state(U0)
    s.advance(100, 0.0, dt0, precision="mixed")
    Umx = s.get_state()
    e = rel_l2(Umx, U64)
    print("vortex 64x64 100 steps mixed vs fp64", e)
    assert e <= 1e-6


def test_mixed_rejects_aliased_buffers():
    torch = pytest.importorskip("torch")
    g = load(NAMES[0])
    s = _solver(g)
    u = torch.from_numpy(g["U0"]).cuda()
    with pytest.raises(ApolloError):
        s.step(0.0, 0.0, u, u, precision="mixed")


def test_mixed_nan_reports_error():
    g = load(NAMES[0])
    s = _solver(g)
    U = g["U0"].copy()
    U[5, 1, 0] = np.nan
    with pytest.raises(ApolloError) as e:
        s.step(0.0, 0.0, U, precision="mixed")
    assert e.value.code == 4


@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_tile_shapes_compute_the_same_steps(N):
    """Both operand chunkings of the chunked mixed stage kernel (shapes 1 and
    2, and shape 0 where the fused kernel does not apply) give the same steps
    bit for bit at any grid share: the same MMAs in the same K order.  The
    fused kernel (shape 0 for four-field Euler at N <= 4) is the same at any
    grid share, and within the mixed form's error of the chunked one."""
    p = problems.euler_vortex(n=17, N=N)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()

    def run(share, shape):
        s.set_launch_shape(share, shape)
        s.set_state(U0)
        t, dt = s.advance(6, 0.0, dt0, precision="mixed")
        return s.get_state(), t, dt

    chunked = [run(1, 2), run(1, 1), run(2, 1), run(4, 2)]
    fused = [run(1, 0), run(4, 0)]
    if N == 5:
        chunked += fused
        fused = []
    for U, t, dt in chunked[1:]:
        np.testing.assert_array_equal(U, chunked[0][0])
        assert t == chunked[0][1] and dt == chunked[0][2]
    for U, t, dt in fused[1:]:
        np.testing.assert_array_equal(U, fused[0][0])
        assert t == fused[0][1] and dt == fused[0][2]
    if fused:
        assert rel_l2(fused[0][0], chunked[0][0]) <= 2e-7
        assert fused[0][1] == pytest.approx(chunked[0][1], rel=1e-7)
    s.set_state(U0)
    s.advance(6, 0.0, dt0)
    assert rel_l2(chunked[0][0], s.get_state()) <= 1e-6
