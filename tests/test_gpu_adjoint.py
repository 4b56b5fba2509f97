"""Derivatives of the float64 path (B200): tangent and discrete adjoint.

The right-hand side's adjoint must be the exact transpose of its tangent
(dot-product test), the tangent must match central finite differences of the
right-hand side, and over a trajectory of fixed SSPRK(5,2) steps the adjoint
gradient of J = 0.5 ||U(T) - U_target||^2 must agree with the tangent
(forward mode) and with central finite differences of J.  The trajectory is
also wrapped as a torch.autograd.Function, as a user of the C ABI would.
"""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import LF_NAMES as NAMES, load

pytestmark = pytest.mark.gpu


def _fixture_solver(g):
    return NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                     numerical_flux=g["numflux"], sources=g["sources"])


@pytest.mark.parametrize("name", NAMES)
def test_rhs_adjoint_is_transpose_of_tangent(name):
    g = load(name)
    s = _fixture_solver(g)
    rng = np.random.default_rng(7)
    x = np.ascontiguousarray(g["U0"])
    v = rng.standard_normal(x.shape)
    w = rng.standard_normal(x.shape)
    jv = s.rhs_jvp(0.25, x, v)
    jtw = s.rhs_vjp(0.25, x, w)
    lhs, rhs = float(np.vdot(w, jv)), float(np.vdot(jtw, v))
    scale = np.linalg.norm(w) * np.linalg.norm(jv) + np.linalg.norm(jtw) * np.linalg.norm(v)
    print(name, lhs, rhs, abs(lhs - rhs) / scale)
    assert abs(lhs - rhs) <= 1e-13 * scale


@pytest.mark.parametrize("name", NAMES)
def test_rhs_tangent_matches_finite_differences(name):
    g = load(name)
    s = _fixture_solver(g)
    rng = np.random.default_rng(3)
    x = np.ascontiguousarray(g["U0"])
    v = rng.standard_normal(x.shape) * (1e-3 * np.abs(x).max())
    # small enough that few face points straddle a switch of the
    # Lax-Friedrichs speed max(c_M, c_P), where the flux has a kink
    eps = 1e-5
    jv = s.rhs_jvp(0.25, x, v)
    rp, _ = s.step(0.25, 0.0, x + eps * v)
    rm, _ = s.step(0.25, 0.0, x - eps * v)
    fd = (rp - rm) / (2 * eps)
    err = np.linalg.norm(fd - jv) / np.linalg.norm(jv)
    print(name, err)
    assert err <= 1e-6


def _vortex_case(n=24, N=3, nsteps=15):
    p = problems.euler_vortex(n=n, N=N)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    u_ic = np.ascontiguousarray(p.ic(x, y))
    s.set_state(u_ic)
    dt = 0.5 * s.init_dt()
    s.forward_fixed(nsteps, 0.0, dt, 4)
    target = s.get_state()
    rng = np.random.default_rng(11)
    u0 = u_ic + 1e-3 * rng.standard_normal(u_ic.shape)
    return s, u0, target, dt, nsteps


def _J(s, u0, target, nsteps, dt, every):
    s.set_state(u0)
    s.forward_fixed(nsteps, 0.0, dt, every)
    uT = s.get_state()
    return 0.5 * float(np.sum((uT - target) ** 2)), uT


def test_trajectory_adjoint_tangent_and_finite_differences():
    s, u0, target, dt, nsteps = _vortex_case()
    J0, uT = _J(s, u0, target, nsteps, dt, 4)
    grad = s.backward(uT - target)
    rng = np.random.default_rng(5)
    for _ in range(4):
        d = rng.standard_normal(u0.shape)
        g_adj = float(np.vdot(grad, d))
        s.set_state(u0)
        duT = s.tangent(nsteps, 0.0, dt, d)
        g_tan = float(np.vdot(uT - target, duT))
        eps = 1e-6
        fd = (_J(s, u0 + eps * d, target, nsteps, dt, 4)[0] - _J(s, u0 - eps * d, target, nsteps, dt, 4)[0]) / (2 * eps)
        print(g_adj, g_tan, fd)
        assert abs(g_adj - g_tan) <= 1e-11 * abs(g_tan)
        assert abs(g_adj - fd) <= 1e-6 * abs(fd)


def test_backward_independent_of_checkpoint_spacing():
    s, u0, target, dt, nsteps = _vortex_case(nsteps=9)
    grads = []
    for every in (1, 4, 9):
        _, uT = _J(s, u0, target, nsteps, dt, every)
        grads.append(s.backward(uT - target))
    for gr in grads[1:]:
        assert np.array_equal(gr, grads[0])
    assert s.adjoint_memory() > 0


def test_boundary_conditions_differentiated():
    # TM walls: the ghost state Ez -> -Ez enters the adjoint through the hook
    p = problems.maxwell_tm(n=10, N=3)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    x, y = s.node_coords()
    u_ic = np.ascontiguousarray(p.ic(x, y))
    s.set_state(u_ic)
    dt = 0.5 * s.init_dt()
    nsteps = 6
    rng = np.random.default_rng(2)
    target = u_ic + 0.01 * rng.standard_normal(u_ic.shape)
    J0, uT = _J(s, u_ic, target, nsteps, dt, 2)
    grad = s.backward(uT - target)
    d = rng.standard_normal(u_ic.shape)
    eps = 1e-6
    fd = (_J(s, u_ic + eps * d, target, nsteps, dt, 2)[0] - _J(s, u_ic - eps * d, target, nsteps, dt, 2)[0]) / (2 * eps)
    assert abs(float(np.vdot(grad, d)) - fd) <= 1e-7 * abs(fd)


def test_torch_autograd_wrapper():
    torch = pytest.importorskip("torch")

    class Trajectory(torch.autograd.Function):
        """U(T) of fixed SSPRK(5,2) steps; backward through apollo_dg_backward."""

        @staticmethod
        def forward(ctx, u0, solver, nsteps, dt, every):
            solver.set_state(u0.detach().contiguous())
            solver.forward_fixed(nsteps, 0.0, dt, every)
            ctx.solver = solver
            return solver.get_state(torch.empty_like(u0))

        @staticmethod
        def backward(ctx, grad_out):
            return ctx.solver.backward(grad_out.contiguous()), None, None, None, None

    s, u0n, targetn, dt, nsteps = _vortex_case(nsteps=10)
    u0 = torch.from_numpy(u0n).cuda().requires_grad_(True)
    target = torch.from_numpy(targetn).cuda()
    loss = 0.5 * ((Trajectory.apply(u0, s, nsteps, dt, 5) - target) ** 2).sum()
    loss.backward()
    g = u0.grad.cpu().numpy()
    d = np.random.default_rng(9).standard_normal(u0n.shape)
    eps = 1e-6
    fd = (_J(s, u0n + eps * d, targetn, nsteps, dt, 5)[0] - _J(s, u0n - eps * d, targetn, nsteps, dt, 5)[0]) / (2 * eps)
    assert abs(float(np.vdot(g, d)) - fd) <= 1e-6 * abs(fd)


def test_trajectory_adjoint_with_hll_flux():
    """The trajectory gradient with Apollo's HLL flux (two-sided faces, wall,
    zero-gradient, inflow and Dirichlet boundaries) agrees with the tangent and
    with central finite differences."""
    from golden_cases import load
    g = load("euler_hll_N3")
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                  numerical_flux="HLL")
    u0 = g["U0"].copy()
    dt = 0.5 * float(g["dt0"])
    nsteps = 4
    s.set_state(u0)
    s.forward_fixed(nsteps, 0.0, dt, 2)
    target = s.get_state() + 1e-3
    J0, uT = _J(s, u0, target, nsteps, dt, 2)
    grad = s.backward(uT - target)
    rng = np.random.default_rng(7)
    for _ in range(3):
        d = rng.standard_normal(u0.shape)
        d[..., 3] = 0.0
        g_adj = float(np.vdot(grad, d))
        s.set_state(u0)
        duT = s.tangent(nsteps, 0.0, dt, d)
        g_tan = float(np.vdot(uT - target, duT))
        eps = 1e-6
        fd = (_J(s, u0 + eps * d, target, nsteps, dt, 2)[0] - _J(s, u0 - eps * d, target, nsteps, dt, 2)[0]) / (2 * eps)
        print(g_adj, g_tan, fd)
        assert abs(g_adj - g_tan) <= 1e-10 * abs(g_tan)
        assert abs(g_adj - fd) <= 1e-5 * abs(fd)


@pytest.mark.parametrize("snapshots", [1, 3, 5, 20])
def test_revolve_gradient_equals_two_level(snapshots):
    """Binomial checkpointing re-runs the same steps with the same kernels, so
    its gradient equals the two-level schedule's bit for bit; the re-run count
    is the host schedule's."""
    s, u0, target, dt, nsteps = _vortex_case(nsteps=23)
    _, uT = _J(s, u0, target, nsteps, dt, 5)
    g2 = s.backward(uT - target)
    s.set_state(u0)
    s.forward_revolve(nsteps, 0.0, dt, snapshots)
    uR = s.get_state()
    assert np.array_equal(uR, uT)
    gr = s.backward(uR - target)
    assert np.array_equal(gr, g2)
    assert s.recomputed_steps() == NodalDG2d.revolve_schedule(nsteps, snapshots)[0]
    # the backward sweep can be repeated on the same trajectory (the first
    # descent is run again: its slots were reused)
    assert np.array_equal(s.backward(uR - target), g2)
    assert s.recomputed_steps() >= NodalDG2d.revolve_schedule(nsteps, snapshots)[0]


def test_revolve_gradient_matches_finite_differences():
    s, u0, target, dt, nsteps = _vortex_case(nsteps=12)

    def J(u):
        s.set_state(u)
        s.forward_revolve(nsteps, 0.0, dt, 4)
        v = s.get_state()
        return 0.5 * float(np.sum((v - target) ** 2)), v

    _, uT = J(u0)
    grad = s.backward(uT - target)
    d = np.random.default_rng(4).standard_normal(u0.shape)
    eps = 1e-6
    fd = (J(u0 + eps * d)[0] - J(u0 - eps * d)[0]) / (2 * eps)
    assert abs(float(np.vdot(grad, d)) - fd) <= 1e-6 * abs(fd)
