"""The oracle's whole right-hand side against Apollo's own (no GPU).

Apollo's WxNodalDG2dMethod, with its geometry (wxnodaldggeometry2d.cc),
cubature (wxcubature2d.cc), node sets and matrices, equation, source and
boundary-condition plugins and limiters, runs compiled unmodified
(oracle/ref_driver.cpp, `make -C oracle refdrv`) over a minimal stand-in for
PETSc's mesh, vector and dense-matrix calls.  Its initial state, initial dt,
right-hand side and suggested dt are compared with the oracle's on the same
mesh and states.  PETSc's dense LU and products go through LAPACK/BLAS, whose
summation order is not known here, so the comparison is to round-off
(1e-12 relative L2; 1e-11 for the isentropic vortex, whose right-hand side is
a small difference of O(1) flux terms), not bit for bit.
"""
import numpy as np
import pytest

from apollo_b200 import problems
from apollo_b200.mesh import jittered_square
from golden_cases import (CHANNEL_DIRICHLET, CHANNEL_INFLOW, channel_mesh, channel_state, one_tag_per_element,
                          rel_l2)

VORTEX = ["r = sqrt((x-xo)*(x-xo)+(y-yo)*(y-yo))", "u = uo - beta*exp(1.-r*r)*(y-yo)/(2.*pi)",
          "v = vo + beta*exp(1.-r*r)*(x-xo)/(2.*pi)",
          "base = 1. - ( (gamma-1.)*beta*beta*exp(2.*(1.-r*r))/(16.*gamma*pi*pi) )", "rho = base^(1./(gamma-1.))",
          "p   = rho^gamma", "en = p/(gamma-1.) + 0.5*rho*(u*u + v*v)", "rhou = rho*u", "rhov = rho*v"]


def _driver(orc, mesh):
    if not orc.RefDriver.available():
        pytest.skip("Apollo's right-hand side is not built here")
    return orc.RefDriver(mesh)


def _deck(N, eq, bcs, meqn, exprs, keys="", progn=None, consts="", blocks=""):
    """A nodalDG2d block as Apollo's example inputs write it (keys first)."""
    pg = "" if progn is None else "  progn = [" + ", ".join(f'"{p}"' for p in progn) + "]\n"
    return (f"<hyperbolic>\n Kind = nodalDG2d\n Equations = [eq]\n boundaryConditions = [{', '.join(bcs)}]\n"
            f" polynomialOrder = {N}\n cfl = 0.5\n DataStructure = [0, dg, {meqn * (N + 1) * (N + 2) // 2}]\n{keys}"
            f" <InitialCondition>\n  Kind = exprFunc\n{consts}  exprList = [" + ", ".join(f'"{e}"' for e in exprs)
            + f"]\n{pg} </InitialCondition>\n{blocks} <eq>\n{eq}\n </eq>\n</hyperbolic>\n")


def _channel(orc, N, code, flux, rotate):
    mesh = one_tag_per_element(channel_mesh(7, seed=N, rotate_seed=rotate))
    bcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, CHANNEL_INFLOW),
           (orc.BC_EULER_DIRICHLET, CHANNEL_DIRICHLET))
    o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0, code), bcs=bcs, cfl=0.5)
    r = _driver(orc, mesh)
    r.add_bc("wall", "eulerWallBC")
    r.add_bc("outflow", "eulerZeroGradientBC")
    r.add_bc("inflow", "eulerInflowBC", **dict(zip(("Mach_number", "Flow_angle", "gas_gamma", "Pressure", "density"),
                                                  CHANNEL_INFLOW)))
    r.add_bc("left", "eulerDirichletBC", **dict(zip(("density", "xvelocity", "yvelocity", "zvelocity", "gas_gamma",
                                                     "pressure"), CHANNEL_DIRICHLET)))
    return mesh, o, r


@pytest.mark.parametrize("N", [2, 3, 4, 5])
@pytest.mark.parametrize("flux", ["LF", "HLL", "Roe", "Wave"])
def test_euler_channel_rhs_vs_reference(oracle_lib, flux, N):
    """Every Euler numerical flux with the wall, zero-gradient, inflow and
    Dirichlet conditions, elements listing their faces in every order."""
    orc = oracle_lib
    code = {"LF": orc.NF_LF, "HLL": orc.NF_HLL, "Roe": orc.NF_ROE, "Wave": orc.NF_WAVE}[flux]
    mesh, o, r = _channel(orc, N, code, flux, rotate=N)
    r.setup(_deck(N, f"  Kind = eulerEqn\n  gas_gamma = 1.4\n  Numerical_Flux = {flux}",
                  ["wall", "outflow", "inflow", "left"], 5, ["1.0", "0.5", "0.1", "0.0", "2.6"]))
    u0, dt0 = r.init(0.0)
    np.testing.assert_array_equal(u0, np.broadcast_to([1.0, 0.5, 0.1, 0.0, 2.6], u0.shape))
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    x, y = o.node_coords()
    for U in (channel_state(x, y), channel_state(x, y, rough=0.05, seed=N)):
        rr, sr = r.rhs(U, 0.3, 0.01)
        ro, so = o.rhs(U, 0.3, 0.01)
        assert o.error == 0
        assert rel_l2(rr, ro) <= 1e-12
        assert sr == pytest.approx(so, rel=1e-14)


@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_isentropic_vortex_vs_reference(oracle_lib, N):
    """Apollo's isentropicVortex example (exprFunc initial state, the exact
    vortex imposed by isentropicVortexBC): the initial state at Apollo's node
    coordinates, the initial dt and the right-hand side."""
    orc = oracle_lib
    mesh = jittered_square(9, (0.0, -5.0), (10.0, 5.0), seed=N, periodic=False, wall_tag=1)
    o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4, 0.0, 0.0), bcs=((orc.BC_VORTEX, (1.0, 0.0, 5.0, 0.0, 1.4, 5.0)),),
                   cfl=0.5)
    r = _driver(orc, mesh)
    r.add_bc("allSides", "isentropicVortexBC", u0=1.0, v0=0.0, x0=5.0, y0=0.0, gas_gamma=1.4, beta=5.0)
    consts = "".join(f"  {k} = {v}\n" for k, v in (("xo", 5.0), ("yo", 0.0), ("beta", 5.0), ("gamma", 1.4),
                                                    ("uo", 1.0), ("vo", 0.0), ("pi", 3.141592653589793)))
    r.setup(_deck(N, "  Kind = eulerEqn\n  gas_gamma = 1.4", ["allSides"], 5, ["rho", "rhou", "rhov", "0.0", "en"],
                  progn=VORTEX, consts=consts))
    u0, dt0 = r.init(0.0)
    x, y = o.node_coords()
    ic = problems.vortex_ic(x, y, 5, x0=5.0, y0=0.0, beta=5.0)
    assert np.abs(u0 - ic).max() <= 1e-13
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    rr, sr = r.rhs(u0, 0.3, 0.01)
    ro, so = o.rhs(u0, 0.3, 0.01)
    assert rel_l2(rr, ro) <= 1e-11
    assert sr == pytest.approx(so, rel=1e-14)


@pytest.mark.parametrize("N", [2, 3, 5])
def test_maxwell_and_sources_vs_reference(oracle_lib, N):
    """phMaxwellEqn: the TM cavity with maxwellTransverseMagneticBC, and the
    cleaned form (chi = gamma = 1) with phmConductingWallBC and both source
    plugins (TM2DwithSource.pin's tranverseMagneticSrc, a pointCurrentSrc)."""
    orc = oracle_lib
    mesh = jittered_square(7, seed=N, periodic=False, wall_tag=1)
    rng = np.random.default_rng(N)
    o = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),), cfl=0.5)
    r = _driver(orc, mesh)
    r.add_bc("walls", "maxwellTransverseMagneticBC")
    r.setup(_deck(N, "  Kind = phMaxwellEqn\n  c0 = 1.0", ["walls"], 8,
                  ["0.0", "0.0", "sin(pi*x)*sin(pi*y)"] + ["0.0"] * 5, consts="  pi = 3.141592653589793\n"))
    u0, dt0 = r.init(0.0)
    x, y = o.node_coords()
    assert np.abs(u0[..., 2] - np.sin(np.pi * x) * np.sin(np.pi * y)).max() <= 1e-15
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    U = rng.standard_normal((mesh.K, x.shape[1], 8))
    assert rel_l2(r.rhs(U, 0.3, 0.01)[0], o.rhs(U, 0.3, 0.01)[0]) <= 1e-12
    pc = (0.4, 0.6, 0.15, 2.0, 5.0, 0.2, 1.0, 2.0, 0.5)
    o = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.0, 1.0, 1.0), bcs=((orc.BC_PEC, ()),), cfl=0.5)
    o.add_source(orc.SRC_TM, 2, ())
    o.add_source(orc.SRC_POINT, 2, pc)
    r = _driver(orc, mesh)
    r.add_bc("walls", "phmConductingWallBC")
    keys = ("xLocation", "yLocation", "radius", "currentDensity", "frequency", "phase", "charge", "mass", "epsilon0")
    blocks = (" <current>\n  Kind = tranverseMagneticSrc\n  OutRange = [2]\n </current>\n <wire>\n"
              "  Kind = pointCurrentSrc\n  OutRange = [2]\n" + "".join(f"  {k} = {v}\n" for k, v in zip(keys, pc))
              + " </wire>\n")
    r.setup(_deck(N, "  Kind = phMaxwellEqn\n  c0 = 1.0\n  chi = 1.0\n  gamma = 1.0", ["walls"], 8, ["0.0"] * 8,
                  keys=" Sources = [current, wire]\n", blocks=blocks))
    for t in (0.3, 1.7):
        rr, ro = r.rhs(U, t, 0.01)[0], o.rhs(U, t, 0.01)[0]
        assert rel_l2(rr, ro) <= 1e-12
    base = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.0, 1.0, 1.0), bcs=((orc.BC_PEC, ()),), cfl=0.5)
    assert rel_l2(base.rhs(U, 0.3, 0.01)[0], o.rhs(U, 0.3, 0.01)[0]) > 1e-4  # the sources were applied


@pytest.mark.parametrize("N", [2, 3, 5])
def test_advection_vs_reference(oracle_lib, N):
    """advectionEqn with a gridFixedBC inflow value."""
    orc = oracle_lib
    mesh = jittered_square(7, seed=N + 10, periodic=False, wall_tag=1)
    o = orc.Oracle(mesh, N, orc.EQ_ADVECTION, (1.0, 0.5, 0.0), bcs=((orc.BC_FIXED, (0.75,)),), cfl=0.5)
    r = _driver(orc, mesh)
    r.add_bc("fixed", "gridFixedBC", value=0.75)
    r.setup(_deck(N, "  Kind = advectionEqn\n  ux = 1.0\n  uy = 0.5", ["fixed"], 1, ["sin(x)*cos(y)"]))
    u0, dt0 = r.init(0.0)
    x, y = o.node_coords()
    assert np.abs(u0[..., 0] - np.sin(x) * np.cos(y)).max() <= 1e-15
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    U = np.random.default_rng(N).standard_normal((mesh.K, x.shape[1], 1))
    rr, sr = r.rhs(U, 0.3, 0.01)
    ro, so = o.rhs(U, 0.3, 0.01)
    assert rel_l2(rr, ro) <= 1e-12
    assert sr == pytest.approx(so, rel=1e-14)


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("kind", ["eulerLimiterHW", "tuAliabadiLimiter"])
def test_limited_rhs_vs_reference(oracle_lib, kind, N):
    """WxNodalDG2dMethod::step with a limiter in its `Limiter` list (the
    limiter acts on the input, then the right-hand side), against the oracle's
    right-hand side of its own limited state."""
    orc = oracle_lib
    floors = (1e-6, 1e-6)
    mesh, o, r = _channel(orc, N, orc.NF_HLL, "HLL", rotate=30 + N)
    eq = "  Kind = eulerEqn\n  gas_gamma = 1.4\n  Numerical_Flux = HLL"
    names = ["wall", "outflow", "inflow", "left"]
    if kind == "eulerLimiterHW":
        o.set_limiter(1.4, *floors)
        r.add_limiter("lim", kind, names, gas_gamma=1.4, min_pressure=floors[0], min_density=floors[1])
    else:
        bcs = ((orc.BC_EULER_WALL, ()), (orc.BC_EULER_ZEROGRAD, ()), (orc.BC_EULER_INFLOW, CHANNEL_INFLOW),
               (orc.BC_EULER_DIRICHLET, CHANNEL_DIRICHLET))
        o = orc.Oracle(mesh, N, orc.EQ_EULER, (1.4,) + floors + (orc.NF_HLL,), bcs=bcs, cfl=0.5)
        o.set_limiter_ta()
        r.add_limiter("lim", kind, names, equation="eulerEqn", gas_gamma=1.4, minPressure=floors[0],
                      minDensity=floors[1])
        eq += f"\n  minPressure = {floors[0]}\n  minDensity = {floors[1]}"
    r.setup(_deck(N, eq, names, 5, ["1.0", "0.5", "0.1", "0.0", "2.6"], keys=" Limiter = [lim]\n"))
    x, y = o.node_coords()
    for U in (channel_state(x, y), channel_state(x, y, rough=0.15, seed=N)):
        rr, _ = r.rhs(U, 0.3, 0.01)
        ro, _ = o.rhs(o.limit(U), 0.3, 0.01)
        assert o.error == 0
        assert rel_l2(rr, ro) <= 1e-12


@pytest.mark.parametrize("name", __import__("golden_cases").APOLLO_NAMES)
def test_oracle_reproduces_apollo_rhs_fixtures(oracle_lib, name):
    """The committed right-hand sides made by Apollo's own code
    (tests/golden/make_apollo_rhs.py) are reproduced by the oracle."""
    from golden_cases import BC_KINDS, SRC_CODES, load_apollo
    orc = oracle_lib
    g = load_apollo(name)
    eq = {"eulerEqn": orc.EQ_EULER, "phMaxwellEqn": orc.EQ_MAXWELL, "advectionEqn": orc.EQ_ADVECTION}[g["equation"]]
    code = {"LF": orc.NF_LF, "HLL": orc.NF_HLL, "Roe": orc.NF_ROE, "Wave": orc.NF_WAVE}[g["numflux"]]
    o = orc.Oracle(g["mesh"], int(g["N"]), eq, tuple(g["eqp"]) + (code,),
                   bcs=tuple((BC_KINDS[n], p) for n, p in g["bcs"]), cfl=0.5)
    for kind, out, params in g["sources"]:
        o.add_source(SRC_CODES[kind], out[0], params)
    U = g["U"]
    if "limiter_kind" in g:  # the limiter acts on the input, then the right-hand side
        if str(g["limiter_kind"]) == "eulerLimiterHW":
            o.set_limiter(*g["limiter"])
        else:
            o.set_limiter_ta()
        U = o.limit(U)
    rhs, sugg = o.rhs(U, float(g["t"]), float(g["dt"]))
    assert rel_l2(rhs, g["rhs"]) <= (1e-11 if "vortex" in name else 1e-12)
    assert sugg == pytest.approx(float(g["sugg"]), rel=1e-14)
    if "steps" in g:  # SSPRK(5,2) steps through Apollo's right-hand side
        U = g["U"].copy()
        n, t, dt = o.run(U, int(g["steps"]), 0.0, float(g["dt"]))
        assert n == int(g["steps"])
        assert rel_l2(U, g["U_end"]) <= 1e-12
        assert t == pytest.approx(float(g["t_end"]), rel=1e-14)
        assert dt == pytest.approx(float(g["dt_end"]), rel=1e-13)


def test_steps_through_apollo_rhs_match_oracle(oracle_lib):
    """SSPRK(5,2) steps with Apollo's dt policy taken through Apollo's own
    right-hand side (what `bench.py --impl reference` times) equal the
    oracle's steps: the isentropicVortex example on a walled square."""
    orc = oracle_lib
    if not orc.RefDriver.available():
        pytest.skip("Apollo's right-hand side is not built here")
    mesh = jittered_square(10, (0.0, 0.0), (10.0, 10.0), seed=2, periodic=False, wall_tag=1)
    r = orc.apollo_vortex_driver(mesh, 4, 0.5)
    u0, dt0 = r.init(0.0)
    o = orc.Oracle(mesh, 4, orc.EQ_EULER, (1.4, 0.0, 0.0), bcs=((orc.BC_VORTEX, (1.0, 0.0, 5.0, 5.0, 1.4, 5.0)),),
                   cfl=0.5)
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    uo = u0.copy()
    n, to, dto = o.run(uo, 4, 0.0, dt0)
    ur, tr, dtr = r.run(u0, 4, 0.0, dt0)
    assert n == 4
    assert rel_l2(ur, uo) <= 1e-12
    assert tr == pytest.approx(to, rel=1e-14) and dtr == pytest.approx(dto, rel=1e-13)


@pytest.mark.parametrize("case", ["tm", "advection"])
def test_example_drivers_step_like_the_oracle(oracle_lib, case):
    """The TM cavity and walled advection problems the bench times through
    Apollo's own code (apollo_tm_driver, apollo_advection_driver) step like
    the oracle on the same problem."""
    orc = oracle_lib
    if not orc.RefDriver.available():
        pytest.skip("Apollo's right-hand side is not built here")
    mesh = jittered_square(8, seed=1, periodic=False, wall_tag=1)
    if case == "tm":
        N, r = 5, orc.apollo_tm_driver(mesh, 5, 0.5)
        o = orc.Oracle(mesh, N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),), cfl=0.5)
    else:
        N, r = 3, orc.apollo_advection_driver(mesh, 3, 0.5)
        o = orc.Oracle(mesh, N, orc.EQ_ADVECTION, (1.0, 0.5, 0.0), bcs=((orc.BC_FIXED, (0.0,)),), cfl=0.5)
    u0, dt0 = r.init(0.0)
    assert dt0 == pytest.approx(o.init_dt(u0), rel=1e-14)
    uo = u0.copy()
    o.run(uo, 3, 0.0, dt0)
    ur, _, _ = r.run(u0, 3, 0.0, dt0)
    assert rel_l2(ur, uo) <= 1e-12
