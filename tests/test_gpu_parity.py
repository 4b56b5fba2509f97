"""CUDA path vs the oracle's golden fixtures and analytic properties (B200)."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import NAMES, load, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, float64 path vs the float64 oracle (states, stage updates)
# The isentropic-vortex RHS is a small difference of O(1) flux terms (the
# far field is a uniform flow whose flux divergence cancels); recompiling the
# oracle itself with FMA contraction moves its RHS by 9e-13 relative L2.  The
# RHS of those fixtures is held to this looser bound, the states to TOL.
RHS_TOL_CANCELLING = 1e-11


def _solver(g):
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                  numerical_flux=g["numflux"], sources=g["sources"])
    if "limiter" in g:
        s.set_limiter(str(g.get("limiter_kind", "eulerLimiterHW")), g["limiter"])
    return s


@pytest.mark.parametrize("name", NAMES)
def test_rhs_matches_oracle(name):
    g = load(name)
    s = _solver(g)
    x, y = s.node_coords()
    assert rel_l2(x, g["x"]) == 0.0
    out, sugg = s.step(0.0, 0.0, g["U0"])
    tol = RHS_TOL_CANCELLING if name.startswith("euler") else TOL
    assert rel_l2(out, g["rhs"]) <= tol
    # the forward-Euler stage u + dt L(u) that the stepper forms
    dt0 = float(g["dt0"])
    assert rel_l2(g["U0"] + dt0 * out, g["U0"] + dt0 * g["rhs"]) <= TOL
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
    host, _ = s.step(0.0, 0.0, g["U0"])
    np.testing.assert_array_equal(out.cpu().numpy(), host)
    tol = RHS_TOL_CANCELLING if name.startswith("euler") else TOL
    assert rel_l2(out.cpu().numpy(), g["rhs"]) <= tol


@pytest.mark.parametrize("case", ["euler5", "euler4", "maxwell8", "maxwell3", "advection"])
@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_rhs_random_states_vs_oracle(case, N):
    """Well-conditioned RHS (random physical states, walls + vortex BC): 1e-12 relative L2."""
    from oracle import oracle as orc
    from apollo_b200.mesh import jittered_square
    rng = np.random.default_rng(100 * N + len(case))
    mesh = jittered_square(7, (0.0, 0.0), (2.0, 1.0), seed=N, periodic=False)
    if case.startswith("euler"):
        m = 5 if case == "euler5" else 4
        kind = "eulerEqn" if m == 5 else "eulerEqn2d"
        vb = (1.0, 0.3, 1.0, 0.5, 1.4, 2.0)
        s = NodalDG2d(N, 0.5, kind, (1.4, 0.0, 0.0), mesh, bcs=(("isentropicVortexBC", vb),))
        o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0), bcs=((orc.BC_VORTEX, vb),))
        # perturbations of a physical state, so that the interpolants at the
        # cubature and Gauss points keep rho > 0 and p > 0
        U = 0.1 * rng.uniform(-1, 1, (mesh.K, s.Np, 5))
        U[..., 0] += 1.0
        U[..., 1] += 0.5
        if m == 4:
            U[..., 3] = 0.0
        U[..., 4] = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2 + U[..., 3] ** 2) / U[..., 0] + 2.0 + U[..., 4]
        sel = [0, 1, 2, 3, 4] if m == 5 else [0, 1, 2, 4]
    elif case.startswith("maxwell"):
        m = 8 if case == "maxwell8" else 3
        if m == 8:
            s = NodalDG2d(N, 0.5, "phMaxwellEqn", (1.3, 0.2, 0.7), mesh, bcs=(("phmConductingWallBC", ()),))
            o = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.3, 0.2, 0.7), bcs=((orc.BC_PEC, ()),))
            U = rng.uniform(-1, 1, (mesh.K, s.Np, 8))
            sel = list(range(8))
        else:
            s = NodalDG2d(N, 0.5, "maxwellTM", (1.3,), mesh, bcs=(("phmConductingWallBC", ()),))
            o = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.3, 0.0, 0.0), bcs=((orc.BC_PEC, ()),))
            U = np.zeros((mesh.K, s.Np, 8))
            U[..., 2:5] = rng.uniform(-1, 1, (mesh.K, s.Np, 3))
            sel = [2, 3, 4]
    else:
        s = NodalDG2d(N, 0.5, "advectionEqn", (0.7, -1.2, 0.0), mesh, bcs=(("gridFixedBC", (0.25,)),))
        o = orc.Oracle(mesh, N, orc.EQ_ADVECTION, (0.7, -1.2, 0.0), bcs=((orc.BC_FIXED, (0.25,)),))
        U = rng.uniform(-1, 1, (mesh.K, s.Np, 1))
        sel = [0]
    ref, sugg_ref = o.rhs(U, 0.3, 0.01)
    out, sugg = s.step(0.3, 0.01, np.ascontiguousarray(U[..., sel]))
    assert rel_l2(out, ref[..., sel]) <= TOL
    assert sugg == pytest.approx(sugg_ref, rel=1e-14)


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
    # relative to the largest integral: the y-momentum integral is ~0 by symmetry
    assert np.all(np.abs(after - before) <= 1e-12 * np.abs(before).max())


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


def _channel_solver(g, kind="eulerEqn", fields=5, flux=None):
    bcs = g["bcs"]
    return NodalDG2d(int(g["N"]), float(g["cfl"]), kind, g["eqp"][:3], g["mesh"], bcs=bcs,
                     numerical_flux=flux or g["numflux"])


@pytest.mark.parametrize("name", ["euler_hll_N3", "euler_roe_N4", "euler_wave_N2"])
def test_planar_euler_equals_full_with_new_fluxes_and_bcs(name):
    """eulerEqn2d equals eulerEqn with rho w = 0 under HLL, Roe and Wave and the
    wall, inflow, zero-gradient and Dirichlet conditions."""
    g = load(name)
    s5 = _channel_solver(g)
    s4 = _channel_solver(g, "eulerEqn2d")
    r5, a5 = s5.step(0.2, 0.01, g["U0"])
    r4, a4 = s4.step(0.2, 0.01, np.ascontiguousarray(g["U0"][..., [0, 1, 2, 4]]))
    assert np.abs(r5[..., 3]).max() == 0.0
    assert rel_l2(r4, r5[..., [0, 1, 2, 4]]) <= 1e-14
    assert a4 == a5


def test_unknown_flux_name_is_lax_friedrichs():
    g = load("euler_hll_N3")
    lf, _ = _channel_solver(g, flux="LF").step(0.0, 0.0, g["U0"])
    other, _ = _channel_solver(g, flux="HLLC").step(0.0, 0.0, g["U0"])
    np.testing.assert_array_equal(other, lf)
    hll, _ = _channel_solver(g).step(0.0, 0.0, g["U0"])
    assert rel_l2(hll, lf) > 1e-3


@pytest.mark.parametrize("name", ["euler_hll_N3", "euler_roe_N4", "euler_wave_N2"])
def test_other_fluxes_adjoint_is_transpose_of_tangent(name):
    """The discrete adjoint of a right-hand side with Apollo's HLL, Roe and
    Wave fluxes (HLL and Wave evaluated from both sides of a face) is the
    transpose of its tangent: <w, J v> = <J^T w, v>."""
    g = load(name)
    s = _solver(g)
    U = g["U0"]
    rng = np.random.default_rng(9)
    v = rng.standard_normal(U.shape)
    w = rng.standard_normal(U.shape)
    v[..., 3] = 0.0
    w[..., 3] = 0.0
    jv = s.rhs_jvp(0.1, U, v)
    jtw = s.rhs_vjp(0.1, U, w)
    lhs, rhs = float(np.vdot(w, jv)), float(np.vdot(jtw, v))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)


def test_hll_tangent_matches_finite_differences():
    """The forward-mode derivative runs through the same templated HLL flux."""
    g = load("euler_hll_N3")
    s = _channel_solver(g)
    U = g["U0"]
    v = np.random.default_rng(5).standard_normal(U.shape)
    v[..., 3] = 0.0
    jv = s.rhs_jvp(0.1, U, v)
    eps = 1e-6
    rp, _ = s.step(0.1, 0.0, U + eps * v)
    rm, _ = s.step(0.1, 0.0, U - eps * v)
    fd = (rp - rm) / (2 * eps)
    assert rel_l2(jv, fd) <= 1e-6


def test_limiter_refusals_and_removal():
    """The limiter is refused where it is not supported, and removing it
    restores the plain right-hand side."""
    from apollo_b200 import ApolloError
    g = load("euler_hll_limiter_N3")
    s = _solver(g)
    with pytest.raises(ApolloError) as e:
        s.rhs_jvp(0.0, g["U0"], g["U0"])
    assert e.value.code == 1
    lim, _ = s.step(0.0, 0.0, g["U0"])
    s.set_limiter(None)
    plain, _ = s.step(0.0, 0.0, g["U0"])
    ref, _ = _channel_solver(g).step(0.0, 0.0, g["U0"])
    np.testing.assert_array_equal(plain, ref)
    assert rel_l2(lim, plain) > 1e-3
    # the vortex boundary condition reads (t, x, y), which the limiter cannot give it
    v = load("euler_gmsh_N3")
    sv = NodalDG2d(int(v["N"]), float(v["cfl"]), v["equation"], v["eqp"][:3], v["mesh"], bcs=v["bcs"])
    with pytest.raises(ApolloError):
        sv.set_limiter("eulerLimiterHW", (1.4, 1e-6, 1e-6))


def test_tu_aliabadi_limiter_kinds():
    """tuAliabadiLimiter: Maxwell nodes become the element averages; on an
    Euler state away from the floors it equals eulerLimiterHW given the
    equation's parameters; advection and explicit parameters are refused."""
    from apollo_b200 import ApolloError
    g = load("maxwell_talimiter_N3")
    s = _solver(g)
    w = s.averaging_weights()
    rng = np.random.default_rng(3)
    U = rng.normal(size=s.shape)
    out, _ = s.step(0.0, 0.0, U)
    s.set_limiter(None)
    avg = np.einsum("n,knm->km", w, U)
    ref, _ = s.step(0.0, 0.0, np.ascontiguousarray(np.broadcast_to(avg[:, None, :], U.shape)))
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    e = load("euler_hll_talimiter_N3")
    a, b = _solver(e), _solver(e)
    b.set_limiter("eulerLimiterHW", tuple(float(v) for v in e["eqp"][:3]))
    ra, rb = a.step(0.0, 0.0, e["U0"])[0], b.step(0.0, 0.0, e["U0"])[0]
    assert rel_l2(ra, rb) <= 1e-14
    with pytest.raises(ApolloError):
        a.set_limiter("tuAliabadiLimiter", (1.4, 1e-6, 1e-6))
    adv = load("adv_N3")
    sa = _solver(adv)
    with pytest.raises(ApolloError):
        sa.set_limiter("tuAliabadiLimiter")


def test_averaging_weights_and_vtu(tmp_path):
    """The averaging weights sum to one and average a linear field to its
    centroid value; the handle writes its state as a VTK frame."""
    from apollo_b200.vtk import read_vtu
    g = load(NAMES[0])
    s = _solver(g)
    w = s.averaging_weights()
    assert abs(w.sum() - 1.0) < 1e-14
    x, y = s.node_coords()
    lin = 2.0 * x - 3.0 * y + 1.0
    verts = g["mesh"].etov
    cx = g["mesh"].vx[verts].mean(axis=1)
    cy = g["mesh"].vy[verts].mean(axis=1)
    np.testing.assert_allclose(lin @ w, 2.0 * cx - 3.0 * cy + 1.0, rtol=0, atol=1e-12)
    s.set_state(g["U0"])
    s.write_vtu(str(tmp_path / "s.vtu"), time=0.0)
    a = read_vtu(str(tmp_path / "s.vtu"))
    np.testing.assert_array_equal(a["solution"], g["U0"].reshape(g["U0"].shape[0], -1))


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("kind", ["eulerLimiterHW", "tuAliabadiLimiter"])
def test_limiter_boundary_face_after_interior_face(N, kind):
    """Apollo's Euler limiters give a boundary face listed after an interior
    face the ghost nodes of the neighbour they read last.  On a channel whose
    elements list their faces in every order (every boundary kind), the B200
    limiter does the same: the right-hand side of the limited state equals the
    oracle's to 1e-12, for smooth and rough states."""
    from oracle import oracle as orc
    from golden_cases import (CHANNEL_DIRICHLET, CHANNEL_INFLOW, boundary_after_interior, channel_mesh,
                              channel_state)
    mesh = channel_mesh(7, seed=N, rotate_seed=10 + N)
    floors = (1e-6, 1e-6)
    bcs = (("eulerWallBC", ()), ("eulerZeroGradientBC", ()), ("eulerInflowBC", CHANNEL_INFLOW),
           ("eulerDirichletBC", CHANNEL_DIRICHLET))
    obcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, CHANNEL_INFLOW),
            (orc.BC_EULER_DIRICHLET, CHANNEL_DIRICHLET))
    eqp = (1.4,) + (floors if kind == "tuAliabadiLimiter" else (0.0, 0.0))
    s = NodalDG2d(N, 0.5, "eulerEqn", eqp, mesh, bcs=bcs, numerical_flux="HLL")
    o = orc.Oracle(mesh, N, orc.EQ_EULER, eqp + (orc.NF_HLL,), bcs=obcs)
    assert boundary_after_interior(o.connectivity(), N) > 0
    if kind == "eulerLimiterHW":
        s.set_limiter(kind, (1.4,) + floors)
        o.set_limiter(1.4, *floors)
    else:
        s.set_limiter(kind)
        o.set_limiter_ta()
    x, y = o.node_coords()
    for U in (channel_state(x, y), channel_state(x, y, rough=0.15, seed=N)):
        got, _ = s.step(0.2, 0.0, U)
        want, _ = o.rhs(o.limit(U), 0.2, 0.0)
        assert o.error == 0
        assert rel_l2(got, want) <= 1e-12
