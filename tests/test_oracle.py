"""The CPU oracle against Apollo's own code and the golden fixtures (no GPU)."""
import numpy as np
import pytest

from apollo_b200 import problems
from apollo_b200.mesh import jittered_square
from golden_cases import (CHANNEL_DIRICHLET, CHANNEL_INFLOW, NAMES, boundary_after_interior, channel_mesh,
                          channel_state, load, rel_l2)


def _ref(orc):
    if not orc.RefPlugins.available():
        pytest.skip("Apollo reference plugins not built here")
    return orc.RefPlugins()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_port_reproduces_golden(oracle_lib, name):
    """The restated plugins reproduce fixtures made with the reference's plugin code."""
    orc = oracle_lib
    g = load(name)
    bcs = tuple((int(k), tuple(g["bc_params"][i]) if "bc_params" in g else ()) for i, k in enumerate(g["bc_kinds"]))
    o = orc.Oracle(g["mesh"], int(g["N"]), int(g["eq"]), g["eqp"], bcs=bcs, cfl=float(g["cfl"]))
    for kind, out, params in g["sources"]:
        o.add_source({"tranverseMagneticSrc": orc.SRC_TM, "pointCurrentSrc": orc.SRC_POINT}[kind], out[0], params)
    x, y = o.node_coords()
    np.testing.assert_array_equal(x, g["x"])
    if "limiter" in g:
        if str(g.get("limiter_kind", "eulerLimiterHW")) == "tuAliabadiLimiter":
            o.set_limiter_ta()
        else:
            o.set_limiter(*g["limiter"])
        rhs, sugg = o.rhs(o.limit(g["U0"]))
    else:
        rhs, sugg = o.rhs(g["U0"])
    assert rel_l2(rhs, g["rhs"]) <= 1e-14
    assert sugg == pytest.approx(float(g["sugg"]), rel=1e-15)
    assert o.init_dt(g["U0"]) == pytest.approx(float(g["dt0"]), rel=1e-15)
    U = g["U0"].copy()
    n, t, dt = o.run(U, int(g["steps"]), 0.0, float(g["dt0"]))
    assert n == int(g["steps"])
    assert rel_l2(U, g["U_end"]) <= 1e-14
    assert t == pytest.approx(float(g["t_end"]), rel=1e-15)


def test_sources_bitexact_vs_reference(oracle_lib):
    """The restated source plugins (tranverseMagneticSrc, pointCurrentSrc)
    equal Apollo's own, compiled unmodified, through its source set
    (WxHyperbolicSrcSet::sourceTerms with OutRange)."""
    orc = oracle_lib
    if not orc.RefPlugins.available():
        pytest.skip("Apollo's plugins are not built on this machine")
    ref = orc.RefPlugins()
    wire = {"OutRange": "[2]", "xLocation": 0.3, "yLocation": 0.6, "radius": 0.2, "currentDensity": 1.5,
            "frequency": 6.0, "phase": 0.3, "charge": 1.0, "mass": 2.0, "epsilon0": 0.5}
    h = ref.sources({"current": ("tranverseMagneticSrc", {"OutRange": "[2]"}), "wire": ("pointCurrentSrc", wire)}, 8)
    from apollo_b200.mesh import jittered_square
    o = orc.Oracle(jittered_square(5, periodic=False), 3, orc.EQ_MAXWELL, (1.0, 1.0, 1.0), bcs=((orc.BC_PEC, ()),))
    o.add_source(orc.SRC_TM, 2)
    o.add_source(orc.SRC_POINT, 2, (0.3, 0.6, 0.2, 1.5, 6.0, 0.3, 1.0, 2.0, 0.5))
    rng = np.random.default_rng(0)
    hits = 0
    for _ in range(2000):
        t, x, y = rng.uniform(0, 2), rng.uniform(0, 1), rng.uniform(0, 1)
        a = ref.source_terms(h, 8, t, x, y)
        np.testing.assert_array_equal(o.source_terms(t, x, y), a)
        hits += (x - 0.3) ** 2 + (y - 0.6) ** 2 < 0.04
    assert hits > 50  # the point current's disc was sampled


def test_plugins_bitexact_vs_reference(oracle_lib):
    """Restated flux / numerical flux / wave speeds equal Apollo's compiled plugins bit for bit."""
    orc = oracle_lib
    ref = _ref(orc)
    rng = np.random.default_rng(7)
    mesh = jittered_square(5, periodic=True)
    for eq, eqp, kind, params, m in [
        (orc.EQ_ADVECTION, (1.0, 0.5, 0.0), "advectionEqn", dict(ux=1.0, uy=0.5), 1),
        (orc.EQ_EULER, (1.4, 0.0, 0.0), "eulerEqn", dict(gas_gamma=1.4), 5),
        (orc.EQ_MAXWELL, (1.3, 0.2, 0.7), "phMaxwellEqn", dict(c0=1.3, gamma=0.2, chi=0.7), 8),
    ]:
        h = ref.equation(kind, **params)
        o = orc.Oracle(mesh, 2, eq, eqp)
        for _ in range(50):
            q = rng.uniform(-1, 1, m)
            if eq == orc.EQ_EULER:
                q[0] = rng.uniform(0.5, 2.0)
                q[4] = 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0] + rng.uniform(0.5, 3.0)
            # one-element RHS of a constant state exercises flux through the oracle
            for d in (0, 1):
                f = ref.flux(h, d, q)
                assert np.all(np.isfinite(f))
            qM, qP = q.copy(), q * rng.uniform(0.9, 1.1, m)
            if eq == orc.EQ_EULER:
                qP[0] = abs(qP[0])
                qP[4] = 0.5 * (qP[1] ** 2 + qP[2] ** 2 + qP[3] ** 2) / qP[0] + 1.0
            nrm = rng.normal(size=2)
            nrm /= np.linalg.norm(nrm)
            fr, lr = ref.numflux(h, nrm, qM, qP)
            U = np.broadcast_to(qM, (mesh.K, 6, m)).copy()
            # the oracle's plugins are exercised through a full RHS below; here
            # compare the reference with the shared device/host physics header
            # through the oracle in reference-plugin mode
            o.use_ref_plugins(ref, h)
            r_ref, s_ref = o.rhs(U)
            o2 = orc.Oracle(mesh, 2, eq, eqp)
            r_port, s_port = o2.rhs(U)
            np.testing.assert_array_equal(r_port, r_ref)
            assert s_port == s_ref
            assert o2.init_dt(U) == o.init_dt(U)
            assert np.isfinite(lr)
            break
        # numerical flux on random pairs via a two-element RHS is covered by the
        # golden fixtures; wave speeds: restated vs reference directly
        if eq != orc.EQ_ADVECTION:
            for _ in range(20):
                q = rng.uniform(-1, 1, m)
                if eq == orc.EQ_EULER:
                    q[0] = rng.uniform(0.5, 2.0)
                    q[4] = 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0] + rng.uniform(0.5, 3.0)
                U = np.broadcast_to(q, (mesh.K, 6, m)).copy()
                o3 = orc.Oracle(mesh, 2, eq, eqp)
                assert o3.init_dt(U) == pytest.approx(
                    2.0 / 3.0 * 0.5 * o3.dtscale * (o3.rmin / np.sqrt(ref.speed2(h, q))), rel=0, abs=0)


def test_rhs_random_states_bitexact(oracle_lib):
    """Full RHS with random (physical) states: port plugins == reference plugins."""
    orc = oracle_lib
    ref = _ref(orc)
    rng = np.random.default_rng(11)
    mesh = jittered_square(6, (0, 0), (2, 1), periodic=False)
    for eq, eqp, kind, params, m, bcs in [
        (orc.EQ_EULER, (1.4, 0.0, 0.0), "eulerEqn", dict(gas_gamma=1.4), 5,
         ((orc.BC_VORTEX, (1.0, 0.0, 1.0, 0.5, 1.4, 2.0)),)),
        (orc.EQ_MAXWELL, (1.3, 0.2, 0.7), "phMaxwellEqn", dict(c0=1.3, gamma=0.2, chi=0.7), 8,
         ((orc.BC_PEC, ()),)),
        (orc.EQ_ADVECTION, (0.7, -1.2, 0.0), "advectionEqn", dict(ux=0.7, uy=-1.2), 1, ((orc.BC_FIXED, (0.25,)),)),
    ]:
        h = ref.equation(kind, **params)
        U = rng.uniform(-1, 1, (mesh.K, 10, m))
        if eq == orc.EQ_EULER:
            U[..., 0] = rng.uniform(0.5, 2.0, U.shape[:2])
            U[..., 4] = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2 + U[..., 3] ** 2) / U[..., 0] + 2.0
        a = orc.Oracle(mesh, 3, eq, eqp, bcs=bcs)
        b = orc.Oracle(mesh, 3, eq, eqp, bcs=bcs)
        b.use_ref_plugins(ref, h)
        ra, sa = a.rhs(U, 0.3, 0.01)
        rb, sb = b.rhs(U, 0.3, 0.01)
        np.testing.assert_array_equal(ra, rb)
        assert sa == sb


@pytest.mark.parametrize("flux", ["HLL", "Roe", "Wave", "LF"])
def test_euler_fluxes_and_bcs_bitexact(oracle_lib, flux):
    """HLL, Roe and Wave restated in the oracle equal Apollo's compiled
    fluxes bit for bit through a full RHS of random states, on a walled mesh
    carrying every Euler boundary condition (wall, inflow, zero gradient,
    Dirichlet)."""
    orc = oracle_lib
    ref = _ref(orc)
    code = {"LF": orc.NF_LF, "HLL": orc.NF_HLL, "Roe": orc.NF_ROE, "Wave": orc.NF_WAVE}[flux]
    rng = np.random.default_rng(23)
    mesh = jittered_square(7, (0, 0), (2, 1), periodic=False, wall_tag=1)
    # tags 1..4 by side: bottom wall, right outflow, top inflow, left Dirichlet
    vn = ((0, 1), (1, 2), (2, 0))
    for f, (i, j) in enumerate(vn):
        ya, yb = mesh.vy[mesh.etov[:, i]], mesh.vy[mesh.etov[:, j]]
        xa, xb = mesh.vx[mesh.etov[:, i]], mesh.vx[mesh.etov[:, j]]
        mesh.face_tag[:, f] = np.select([(ya == 0) & (yb == 0), (xa == 2) & (xb == 2), (ya == 1) & (yb == 1),
                                         (xa == 0) & (xb == 0)], [1, 2, 3, 4], 0)
    bcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, (0.8, 30.0, 1.4, 1.0, 1.2)),
           (orc.BC_EULER_DIRICHLET, (0.9, 0.5, -0.2, 0.0, 1.4, 0.8)))
    h = ref.equation("eulerEqn", gas_gamma=1.4, Numerical_Flux=flux)
    eqp = (1.4, 0.0, 0.0, code)
    for trial in range(3):
        U = rng.uniform(-1, 1, (mesh.K, 10, 5))
        U[..., 0] = rng.uniform(0.5, 2.0, U.shape[:2])
        U[..., 3] = 0.0
        U[..., 4] = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2) / U[..., 0] + rng.uniform(1.0, 3.0, U.shape[:2])
        a = orc.Oracle(mesh, 3, orc.EQ_EULER, eqp, bcs=bcs)
        b = orc.Oracle(mesh, 3, orc.EQ_EULER, eqp, bcs=bcs)
        b.use_ref_plugins(ref, h)
        ra, sa = a.rhs(U, 0.3, 0.01)
        rb, sb = b.rhs(U, 0.3, 0.01)
        assert a.error == 0 and b.error == 0
        np.testing.assert_array_equal(ra, rb)
        assert sa == sb
    if flux == "Roe":
        # Apollo's Roe flux leaves the y-momentum component at zero
        f, _ = ref.numflux(h, np.array([0.6, 0.8]), U[0, 0], U[1, 0])
        assert f[2] == 0.0 and f[3] == 0.0


@pytest.mark.parametrize("prob,text,fields", [
    ("vortex", """<ic>
 xo = 5.
 yo = 5.
 beta = 5.
 gamma = 1.4
 uo = 1.
 vo = 0.
 pi = 3.141592653589793
 exprList = ["rho","rhou","rhov","0.0","en"]
 progn = ["r = sqrt((x-xo)*(x-xo)+(y-yo)*(y-yo))", "u = uo - beta*exp(1.-r*r)*(y-yo)/(2.*pi)", "v = vo + beta*exp(1.-r*r)*(x-xo)/(2.*pi)", "base = 1. - ( (gamma-1.)*beta*beta*exp(2.*(1.-r*r))/(16.*gamma*pi*pi) )", "rho = base^(1./(gamma-1.))", "p   = rho^gamma", "en = p/(gamma-1.) + 0.5*rho*(u*u + v*v)", "rhou = rho*u", "rhov = rho*v"]
</ic>""", 5),
    ("tm", """<ic>
 pi = 3.141592653589793
 exprList = ["0.0", "0.0", "Ez", "0.0", "0.0", "0.0", "0.0", "0.0"]
 progn = ["Ez = sin(pi*x)*sin(pi*y)"]
</ic>""", 8),
])
def test_initial_conditions_vs_reference_exprfunc(oracle_lib, prob, text, fields):
    """The closed-form initial states equal Apollo's exprFunc on the example inputs' expressions."""
    orc = oracle_lib
    ref = _ref(orc)
    h = ref.exprfunc(text)
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 10 if prob == "vortex" else 1, (40, 2))
    for x, y in pts:
        want = ref.exprfunc_eval(h, 0.0, x, y)
        if prob == "vortex":
            got = problems.vortex_ic(np.array([x]), np.array([y]), fields=5)[0]
        else:
            got = problems.tm_ic(np.array([x]), np.array([y]), fields=8)[0]
        np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-15)


def test_conservation_periodic(oracle_lib):
    """On a periodic mesh the element integrals of the RHS sum to zero per field."""
    orc = oracle_lib
    prob = problems.euler_vortex(n=9, N=3, fields=5)
    o = orc.Oracle(prob.mesh, 3, orc.EQ_EULER, (1.4, 0, 0), cfl=0.5)
    x, y = o.node_coords()
    U = prob.ic(x, y)
    rhs, _ = o.rhs(U)
    VVT = o.operator(4)
    w = np.linalg.inv(VVT).sum(axis=0)  # integrals of the nodal basis
    # J per element from the vertex coordinates
    m = prob.mesh
    p = np.stack([m.vx[m.etov], m.vy[m.etov]], -1)
    J = 0.25 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    tot = np.einsum("k,j,kjf->f", J, w, rhs)
    scale = np.einsum("k,j,kjf->f", J, w, np.abs(rhs))
    assert np.all(np.abs(tot) <= 1e-12 * np.maximum(scale, 1.0))


def test_tu_aliabadi_pieces_bitexact_vs_reference(oracle_lib):
    """The Tu-Aliabadi limiter's equation hooks restated in the oracle (Euler
    primitive variables with their floors, which rewrite the conserved input,
    and one node's reconstruction) equal Apollo's compiled eulerEqn plugin bit
    for bit, on states that do and do not reach the floors."""
    orc = oracle_lib
    ref = _ref(orc)
    rng = np.random.default_rng(11)
    minP, minD = 1e-3, 1e-2
    h = ref.equation("eulerEqn", gas_gamma=1.4, minPressure=minP, minDensity=minD)
    mesh = jittered_square(4, (0.0, 0.0), (1.0, 1.0), jitter=0.1, seed=1, periodic=True)
    o = orc.Oracle(mesh, 2, orc.EQ_EULER, (1.4, minP, minD))
    o.set_limiter_ta()
    for trial in range(400):
        q = rng.uniform(-1, 1, 5)
        q[0] = rng.uniform(-0.2, 2.0)           # some at or below zero density
        q[4] = rng.uniform(-0.5, 3.0)           # some with negative pressure
        if abs(q[0]) < 1e-9:
            q[0] = 0.5
        ca, pa = o.ta_prim(q)
        cb, pb = ref.primitive(h, q)
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(pa, pb)
    for trial in range(400):
        rho = rng.uniform(0.05, 2.0)
        u = rng.uniform(-1, 1, 3)
        p = rng.uniform(0.01, 2.0)
        cp = np.array([rho, u[0], u[1], u[2], p])
        cc = np.array([rho, rho * u[0], rho * u[1], rho * u[2], p / 0.4 + 0.5 * rho * (u @ u)])
        # deviations large enough to reach the density and pressure fixes now and then
        dq = rng.normal(0, 1, 5) * np.array([rho, 0.5, 0.5, 0.5, p]) * rng.choice([0.1, 1.0, 3.0])
        out, err = o.ta_node(cc, cp, dq)
        if err or out[0] <= 0 or not np.all(np.isfinite(out)):
            continue  # Apollo's plugin exits the process on these
        np.testing.assert_array_equal(out, ref.ta_limit(h, cc, cp, dq))


def test_tu_aliabadi_equals_hw_without_floors(oracle_lib):
    """Away from the floors the two Euler limiters compute the same state."""
    orc = oracle_lib
    g = load("euler_hll_talimiter_N3")
    bcs = tuple((int(k), tuple(g["bc_params"][i])) for i, k in enumerate(g["bc_kinds"]))
    a = orc.Oracle(g["mesh"], int(g["N"]), int(g["eq"]), g["eqp"], bcs=bcs)
    b = orc.Oracle(g["mesh"], int(g["N"]), int(g["eq"]), g["eqp"], bcs=bcs)
    a.set_limiter_ta()
    b.set_limiter(float(g["eqp"][0]), float(g["eqp"][1]), float(g["eqp"][2]))
    la, lb = a.limit(g["U0"]), b.limit(g["U0"])
    assert not np.array_equal(la, g["U0"])
    np.testing.assert_array_equal(la, lb)


def _reflim(orc, o):
    if not orc.RefLimiter.available():
        pytest.skip("Apollo reference limiter not built here")
    return orc.RefLimiter(o)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_euler_limiter_hw_bitexact_vs_reference(oracle_lib, N):
    """The oracle's eulerLimiterHW restatement equals Apollo's limiter code
    (wxhesthavenwarburtoneulerlimiter.cc, compiled unmodified with its four
    Euler boundary-condition plugins) bit for bit, on a channel with every
    boundary kind whose elements list their faces in every order (a boundary
    face after an interior one takes its ghost nodes from the neighbour Apollo
    read last), for smooth and rough states and with floors high enough that
    the density and pressure fix-ups run."""
    orc = oracle_lib
    mesh = channel_mesh(7, seed=N, rotate_seed=10 + N)
    bcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, CHANNEL_INFLOW),
           (orc.BC_EULER_DIRICHLET, CHANNEL_DIRICHLET))
    o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0, orc.NF_HLL), bcs=bcs)
    assert boundary_after_interior(o.connectivity(), N) > 0
    r = _reflim(orc, o)
    r.add_bc("wall", "eulerWallBC")
    r.add_bc("outflow", "eulerZeroGradientBC")
    r.add_bc("inflow", "eulerInflowBC", **dict(zip(("Mach_number", "Flow_angle", "gas_gamma", "Pressure", "density"),
                                                  CHANNEL_INFLOW)))
    r.add_bc("left", "eulerDirichletBC", **dict(zip(("density", "xvelocity", "yvelocity", "zvelocity", "gas_gamma",
                                                     "pressure"), CHANNEL_DIRICHLET)))
    x, y = o.node_coords()
    smooth, rough = channel_state(x, y), channel_state(x, y, rough=0.15, seed=40 + N)
    fired = False
    for floors in ((1e-6, 1e-6), (1.2, 1.05)):
        o.set_limiter(1.4, *floors)
        r.set_limiter(["wall", "outflow", "inflow", "left"], 1.4, *floors)
        for U in (smooth, rough):
            a, b = o.limit(U), r.limit(U)
            np.testing.assert_array_equal(a, b)
            if floors[0] > 1:
                o.set_limiter(1.4, 1e-6, 1e-6)
                fired |= not np.array_equal(a, o.limit(U))
                o.set_limiter(1.4, *floors)
    assert fired  # the high floors changed the reconstruction


def test_boundary_conditions_bitexact_vs_reference(oracle_lib):
    """Each boundary condition restated in the oracle equals Apollo's plugin
    (compiled unmodified) at random points, times, normals and states:
    gridFixedBC, isentropicVortexBC, the four Euler conditions,
    maxwellTransverseMagneticBC and phmConductingWallBC."""
    orc = oracle_lib
    rng = np.random.default_rng(77)
    mesh = jittered_square(5, periodic=False)
    vortex = (1.0, 0.3, 5.0, 4.0, 1.4, 5.0)
    inflow = (0.8, 30.0, 1.4, 1.0, 1.2)
    dirichlet = (0.9, 0.5, -0.2, 0.1, 1.4, 0.8)
    cases = [  # oracle equation, its bcs, Apollo kind per tag with its keys
        (orc.EQ_ADVECTION, (1.0, 0.5, 0.0), ((orc.BC_FIXED, (0.75,)),), [("gridFixedBC", dict(value=0.75))], 1),
        (orc.EQ_EULER, (1.4, 0.0, 0.0),
         ((orc.BC_VORTEX, vortex), (orc.BC_EULER_WALL, ()), (orc.BC_EULER_INFLOW, inflow),
          (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_DIRICHLET, dirichlet)),
         [("isentropicVortexBC", dict(zip(("u0", "v0", "x0", "y0", "gas_gamma", "beta"), vortex))),
          ("eulerWallBC", {}),
          ("eulerInflowBC", dict(zip(("Mach_number", "Flow_angle", "gas_gamma", "Pressure", "density"), inflow))),
          ("eulerZeroGradientBC", {}),
          ("eulerDirichletBC", dict(zip(("density", "xvelocity", "yvelocity", "zvelocity", "gas_gamma", "pressure"),
                                        dirichlet)))], 5),
        (orc.EQ_MAXWELL, (1.0, 1.0, 1.0), ((orc.BC_TM, ()), (orc.BC_PEC, ())),
         [("maxwellTransverseMagneticBC", {}), ("phmConductingWallBC", {})], 8),
    ]
    for eq, eqp, bcs, kinds, m in cases:
        o = orc.Oracle(mesh, 3, eq, eqp, bcs=bcs)
        r = _reflim(orc, o)
        for tag, (kind, keys) in enumerate(kinds, start=1):
            r.add_bc(f"bc{tag}", kind, **keys)
            for _ in range(50):
                xc = (rng.uniform(0, 2), rng.uniform(0, 10), rng.uniform(0, 10))
                th = rng.uniform(0, 2 * np.pi)
                nx = (np.cos(th), np.sin(th))
                q = rng.uniform(-1, 1, m)
                if m == 5:
                    q[0] = rng.uniform(0.5, 2.0)
                    q[4] = 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0] + rng.uniform(1.0, 3.0)
                a, b = o.apply_bc(tag, xc, nx, q), r.apply_bc(f"bc{tag}", xc, nx, q)
                if kind == "gridFixedBC":  # Apollo writes the one advected field only
                    a, b = a[:1], b[:1]
                np.testing.assert_array_equal(a, b, err_msg=kind)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_tu_aliabadi_limiter_bitexact_vs_reference(oracle_lib, N):
    """The oracle's tuAliabadiLimiter restatement equals Apollo's limiter code
    (aptualiabadilimiter.cc over the eulerEqn and phMaxwellEqn plugins,
    compiled unmodified) bit for bit: the Euler channel with every boundary
    kind and faces in every order, with the equation's floors low and high,
    and the Maxwell TM cavity with its walls."""
    orc = oracle_lib
    mesh = channel_mesh(7, seed=N, rotate_seed=20 + N)
    bcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, CHANNEL_INFLOW),
           (orc.BC_EULER_DIRICHLET, CHANNEL_DIRICHLET))
    names = ["wall", "outflow", "inflow", "left"]
    for floors in ((1e-6, 1e-6), (1.2, 1.05)):
        o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4,) + floors + (orc.NF_HLL,), bcs=bcs)
        assert boundary_after_interior(o.connectivity(), N) > 0
        o.set_limiter_ta()
        r = _reflim(orc, o)
        r.add_bc("wall", "eulerWallBC")
        r.add_bc("outflow", "eulerZeroGradientBC")
        r.add_bc("inflow", "eulerInflowBC", **dict(zip(("Mach_number", "Flow_angle", "gas_gamma", "Pressure",
                                                        "density"), CHANNEL_INFLOW)))
        r.add_bc("left", "eulerDirichletBC", **dict(zip(("density", "xvelocity", "yvelocity", "zvelocity",
                                                         "gas_gamma", "pressure"), CHANNEL_DIRICHLET)))
        r.set_limiter_ta(names, "eulerEqn", gas_gamma=1.4, minPressure=floors[0], minDensity=floors[1])
        x, y = o.node_coords()
        for U in (channel_state(x, y), channel_state(x, y, rough=0.15, seed=50 + N)):
            np.testing.assert_array_equal(o.limit(U), r.limit(U))
    p = problems.maxwell_tm(n=6, N=N, fields=8, seed=N)
    o = orc.Oracle(p.mesh, N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),))
    o.set_limiter_ta()
    r = _reflim(orc, o)
    r.add_bc("walls", "maxwellTransverseMagneticBC")
    r.set_limiter_ta(["walls"], "phMaxwellEqn", c0=1.0)
    x, y = o.node_coords()
    U = np.ascontiguousarray(p.ic(x, y)) + 0.1 * np.random.default_rng(N).standard_normal((p.mesh.K, x.shape[1], 8))
    np.testing.assert_array_equal(o.limit(U), r.limit(U))
