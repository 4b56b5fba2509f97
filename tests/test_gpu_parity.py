"""CUDA path vs the oracle's golden fixtures and analytic properties (B200)."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import NAMES, load, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, float64 path vs the float64 oracle


def _solver(g):
    return NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"])


@pytest.mark.parametrize("name", NAMES)
def test_rhs_matches_oracle(name):
    g = load(name)
    s = _solver(g)
    x, y = s.node_coords()
    assert rel_l2(x, g["x"]) == 0.0
    out, sugg = s.step(0.0, 0.0, g["U0"])
    assert rel_l2(out, g["rhs"]) <= TOL
    assert sugg == pytest.approx(float(g["sugg"]), rel=1e-14)


@pytest.mark.parametrize("name", NAMES)
def test_steps_match_oracle(name):
    g = load(name)
    s = _solver(g)
    s.set_state(g["U0"])
    dt0 = s.init_dt()
    assert dt0 == pytest.approx(float(g["dt0"]), rel=1e-14)
    t, dt = s.advance(int(g["steps"]), 0.0, dt0)
    U = s.get_state()
    assert rel_l2(U, g["U_end"]) <= TOL
    assert t == pytest.approx(float(g["t_end"]), rel=1e-14)
    assert dt == pytest.approx(float(g["dt_end"]), rel=1e-13)


@pytest.mark.parametrize("name", NAMES)
def test_device_pointers(name):
    torch = pytest.importorskip("torch")
    g = load(name)
    s = _solver(g)
    u = torch.from_numpy(g["U0"]).cuda()
    out = torch.empty_like(u)
    s.step(0.0, 0.0, u, out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), g["rhs"]) <= TOL


def test_reduced_fields_equal_full_fields():
    """eulerEqn2d (4 fields) equals eulerEqn (5 fields) with rho w = 0; maxwellTM equals phMaxwellEqn."""
    p5 = problems.euler_vortex(n=9, N=4, fields=5)
    p4 = problems.euler_vortex(n=9, N=4, fields=4)
    s5 = NodalDG2d(4, 0.5, p5.equation, p5.eq_params, p5.mesh)
    s4 = NodalDG2d(4, 0.5, p4.equation, p4.eq_params, p4.mesh)
    x, y = s5.node_coords()
    r5, a5 = s5.step(0.0, 0.0, np.ascontiguousarray(p5.ic(x, y)))
    r4, a4 = s4.step(0.0, 0.0, np.ascontiguousarray(p4.ic(x, y)))
    assert np.abs(r5[..., 3]).max() == 0.0
    assert rel_l2(r4, r5[..., [0, 1, 2, 4]]) <= 1e-14
    assert a4 == a5
    m8 = problems.maxwell_tm(n=7, N=3, fields=8)
    m3 = problems.maxwell_tm(n=7, N=3, fields=3)
    s8 = NodalDG2d(3, 0.5, m8.equation, m8.eq_params, m8.mesh, bcs=m8.bcs)
    s3 = NodalDG2d(3, 0.5, m3.equation, m3.eq_params, m3.mesh, bcs=m3.bcs)
    x, y = s8.node_coords()
    r8, _ = s8.step(0.0, 0.0, np.ascontiguousarray(m8.ic(x, y)))
    r3, _ = s3.step(0.0, 0.0, np.ascontiguousarray(m3.ic(x, y)))
    assert rel_l2(r3, r8[..., [2, 3, 4]]) <= 1e-14


def test_conservation_full_size_periodic():
    """Config-2 size: per-field element integrals are conserved by the stepper (periodic mesh)."""
    p = problems.euler_vortex()
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    s.set_state(np.ascontiguousarray(p.ic(x, y)))
    before = s.integrals()
    dt0 = s.init_dt()
    s.advance(20, 0.0, dt0)
    after = s.integrals()
    assert np.all(np.abs(after - before) <= 1e-11 * np.abs(before))


def test_nan_input_reports_error():
    from apollo_b200 import ApolloError
    g = load(NAMES[0])
    s = _solver(g)
    U = g["U0"].copy()
    U[3, 2, 0] = np.nan
    with pytest.raises(ApolloError) as e:
        s.step(0.0, 0.0, U)
    assert e.value.code == 4


def test_negative_density_reports_error():
    from apollo_b200 import ApolloError
    p = problems.euler_vortex(n=6, N=3, fields=5)
    s = NodalDG2d(3, 0.5, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U = np.ascontiguousarray(p.ic(x, y))
    U[2, :, 0] = -1.0
    with pytest.raises(ApolloError) as e:
        s.step(0.0, 0.0, U)
    assert e.value.code == 3
