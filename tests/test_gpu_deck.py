"""Handles configured from Apollo input-deck text through the C ABI
(apollo_dg_set_equation_text, apollo_dg_add_bc_text, apollo_dg_set_limiter_text)
compute what handles configured with the numeric calls compute, and reproduce
the oracle's golden fixtures (B200)."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d
from apollo_b200.deck import solver_from_deck
from golden_cases import load, rel_l2

pytestmark = pytest.mark.gpu

EQ_KEYS = {"eulerEqn": ("gas_gamma", "minPressure", "minDensity"), "phMaxwellEqn": ("c0", "gamma", "chi"),
           "advectionEqn": ("ux", "uy", "uz")}
BC_KEYS = {"gridFixedBC": ("value",), "isentropicVortexBC": ("u0", "v0", "x0", "y0", "gas_gamma", "beta"),
           "eulerInflowBC": ("Mach_number", "Flow_angle", "gas_gamma", "Pressure", "density"),
           "eulerDirichletBC": ("density", "xvelocity", "yvelocity", "zvelocity", "gas_gamma", "pressure")}


def deck_for(g):
    """An input deck in Apollo's layout for a golden fixture."""
    kind = g["equation"]
    eq = "\n".join(f"      {k} = {float(v)!r}" for k, v in zip(EQ_KEYS[kind], g["eqp"][:3]))
    names = [f"bc{i}" for i in range(len(g["bcs"]))]
    blocks = []
    for nm, (bk, bp) in zip(names, g["bcs"]):
        keys = "\n".join(f"    {k} = {float(v)!r}" for k, v in zip(BC_KEYS.get(bk, ()), bp))
        blocks.append(f"  <{nm}>\n    Type = ApSubSolver\n    Kind = {bk}\n{keys}\n  </{nm}>")
    flux = f"      Numerical_Flux = {g['numflux']}\n" if kind == "eulerEqn" else ""
    SRC_KEYS = ("xLocation", "yLocation", "radius", "currentDensity", "frequency", "phase", "charge", "mass",
                "epsilon0")
    snames = [f"src{i}" for i in range(len(g["sources"]))]
    for nm, (sk, out, sp) in zip(snames, g["sources"]):
        keys = "".join(f"    {k} = {float(v)!r}\n" for k, v in zip(SRC_KEYS, sp))
        blocks.append(f"  <{nm}>\n    Type = WxHyperbolicSrc\n    Kind = {sk}\n    OutRange = [{out[0]}]\n{keys}  </{nm}>")
    srcline = f"Sources = [{', '.join(snames)}]" if snames else ""
    lim = ""
    if "limiter" in g:
        lk = str(g.get("limiter_kind", "eulerLimiterHW"))
        lp = "".join(f"    {k} = {float(v)!r}\n" for k, v in zip(("gas_gamma", "min_pressure", "min_density"), g["limiter"]))
        lim = f"  <lim>\n    Type = ApSubSolver\n    Kind = {lk}\n{lp if lk == 'eulerLimiterHW' else ''}  </lim>\n"
    return f"""# -*- python -*-
ORDER = {int(g['N'])}
<warpx>
 <sim>
   <hyperbolic>
     Type = ApSubSolver
     Kind = nodalDG2d
     Equations = [eq]
     boundaryConditions = [{', '.join(names)}]
     {'Limiter = [lim]' if lim else ''}
     {srcline}
     polynomialOrder = ORDER
     cfl = {float(g['cfl'])!r}
     <eq>
      Type = WxHyperbolicEqn
      Kind = {kind}
{eq}
{flux}     </eq>
   </hyperbolic>
{chr(10).join(blocks)}
{lim} </sim>
</warpx>
"""


@pytest.mark.parametrize("name", ["euler_N4", "euler_hll_N3", "euler_hll_limiter_N3", "maxwell_N5", "adv_N3",
                                  "maxwell_src_N3"])
def test_deck_configured_handle_matches(name):
    g = load(name)
    text = deck_for(g)
    s = solver_from_deck(text, g["mesh"])
    ref = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                    numerical_flux=g["numflux"], sources=g["sources"])
    if "limiter" in g:
        ref.set_limiter(str(g.get("limiter_kind", "eulerLimiterHW")), g["limiter"])
    a, sa = s.step(0.0, 0.0, g["U0"])
    b, sb = ref.step(0.0, 0.0, g["U0"])
    np.testing.assert_array_equal(a, b)
    assert sa == sb
    assert rel_l2(a, g["rhs"]) <= (1e-11 if name.startswith("euler") else 1e-12)
    s.set_state(g["U0"])
    dt0 = s.init_dt()
    s.advance(int(g["steps"]), 0.0, dt0)
    assert rel_l2(s.get_state(), g["U_end"]) <= 1e-12
