"""Apollo input-deck text through the C ABI's host-only deck calls (no GPU):
the sub-solver's order and cfl, the equation block with its numerical flux,
the boundary-condition list and the limiter, with Apollo's key names and
defaults; Apollo's own example decks where the reference tree is present."""
import os

import pytest

from apollo_b200 import ApolloError
from apollo_b200.deck import deck_bcs, deck_config, deck_equation, deck_limiter

DECK = """# -*- python -*-
import math
PI = math.pi
P_ORDER = 3
GAMMA = 1.4
<warpx>
 Simulation = run
 <run>
   Type = WxSolver
   Kind = comboSolver
   <hyperbolic>
     Type = ApSubSolver
     Kind = nodalDG2d
     Equations = [gas]
     boundaryConditions = [left, walls, walls, out]   # tags 1..4
     Limiter = [lim]
     polynomialOrder = P_ORDER
     cfl = 0.9/((2.*(P_ORDER+1)-1))
     exprList = ["rho", \\
                 "0.0"]
     <gas>
       Type = WxHyperbolicEqn
       Kind = eulerEqn
       gas_gamma = GAMMA
       minPressure = 1.e-3
       Numerical_Flux = "Roe"
     </gas>
   </hyperbolic>
   <left>
     Type = ApSubSolver
     Kind = eulerInflowBC
     Mach_number = 2.0
     Flow_angle = 0.0
     gas_gamma = GAMMA
     Pressure = 1.0/GAMMA
     density = 1.0
   </left>
   <walls>
     Type = ApSubSolver
     Kind = eulerWallBC
   </walls>
   <out>
     Type = ApSubSolver
     Kind = eulerZeroGradientBC
   </out>
   <lim>
     Type = ApSubSolver
     Kind = eulerLimiterHW
     gas_gamma = GAMMA
     min_pressure = 2**-7
     min_density = 1e-2
     boundaryConditions = [left]
   </lim>
 </run>
</warpx>
"""


def test_deck_sub_solver_values():
    N, cfl = deck_config(DECK)
    assert N == 3 and cfl == pytest.approx(0.9 / 7.0, rel=1e-15)
    kind, params, flux = deck_equation(DECK)
    assert kind == "eulerEqn" and flux == "Roe"
    assert params == (1.4, 1e-3, 0.0)  # minDensity defaults to 0 as in Apollo
    bcs = deck_bcs(DECK)
    assert [b[0] for b in bcs] == ["eulerInflowBC", "eulerWallBC", "eulerWallBC", "eulerZeroGradientBC"]
    assert bcs[0][1] == pytest.approx((2.0, 0.0, 1.4, 1.0 / 1.4, 1.0), rel=1e-15)
    assert deck_limiter(DECK) == ("eulerLimiterHW", (1.4, 2.0 ** -7, 1e-2))


def test_deck_single_blocks_with_kind():
    assert deck_equation("ux = 1.0\nuy = 0.5", kind="advectionEqn") == ("advectionEqn", (1.0, 0.5, 0.0), "LF")
    assert deck_equation("<m>\n c0 = 2\n chi = 0.5\n</m>", kind="phMaxwellEqn")[1] == (2.0, 0.0, 0.5)
    assert deck_bcs("value = -0.25", kind="gridFixedBC") == [("gridFixedBC", (-0.25,))]
    assert deck_limiter("", kind="tuAliabadiLimiter") == ("tuAliabadiLimiter", ())
    # a single block without a list: its Kind decides
    assert deck_equation("<e>\n Kind = maxwellTM\n c0 = 1\n</e>")[0] == "maxwellTM"


@pytest.mark.parametrize("text, what", [
    ("<gas>\n Kind = eulerEqn\n</gas>", "missing gas_gamma"),
    ("<gas>\n Kind = nosuchEqn\n</gas>", "unknown Kind"),
    ("<gas>\n Kind = eulerEqn\n gas_gamma = LIGHT\n</gas>", "not a number"),
    ("<a>\n Kind = eulerEqn\n</b>", "unbalanced"),
    ("<a>\n Kind = eulerEqn\n", "not closed"),
    ("<s>\n Equations = [a, b]\n <a>\n Kind = eulerEqn\n gas_gamma = 1.4\n </a>\n</s>", "more than one"),
    ("<s>\n Equations = [missing]\n</s>", "no block"),
])
def test_deck_errors(text, what):
    with pytest.raises(ApolloError) as e:
        deck_equation(text)
    assert e.value.code == 1  # APOLLO_ERR_CONFIG
    assert what in str(e.value)


def _examples():
    from oracle.oracle import reference_src
    return os.path.join(reference_src(), "..", "examples", "unstructuredDG")


@pytest.mark.skipif(not os.path.isdir(_examples()), reason="Apollo's example decks are not on this machine")
@pytest.mark.parametrize("deck, N, eq, flux, bcs, lim", [
    ("euler/isentropicVortex/isentropicVortex.pin", 1, ("eulerEqn", (1.4, 0.0, 0.0)), "LF",
     [("isentropicVortexBC", (1.0, 0.0, 5.0, 0.0, 1.4, 5.0))], None),
    ("maxwell/transverseMagnetic/transverseMagnetic.pin", 2, ("phMaxwellEqn", (1.0, 0.0, 0.0)), "LF",
     [("maxwellTransverseMagneticBC", ())], None),
    ("euler/forwardFacingStep/HLLflux/forwardFacingStep.pin", 1, ("eulerEqn", (1.4, 0.0, 0.0)), "HLL",
     [("eulerInflowBC", (3.0, 0.0, 1.4, 5.0, 1.4)), ("eulerWallBC", ()), ("eulerWallBC", ()),
      ("eulerZeroGradientBC", ())], ("eulerLimiterHW", (1.4, 0.01, 0.01))),
    ("advection/advection.pin", 1, ("advectionEqn", (-1.0, -1.0, 0.0)), "LF", [("gridFixedBC", (0.0,))] * 4, None),
])
def test_apollo_example_decks(deck, N, eq, flux, bcs, lim):
    text = open(os.path.join(_examples(), deck)).read()
    assert deck_config(text)[0] == N
    kind, params, nf = deck_equation(text)
    assert (kind, params) == eq and nf == flux
    assert deck_bcs(text) == bcs
    assert deck_limiter(text) == lim


def test_keys_after_a_sub_block_are_not_read_as_in_apollo(oracle_lib):
    """Apollo's cryptset reader does not see a key written after a sub-block
    of the same block: Numerical_Flux = HLL there leaves the Lax-Friedrichs
    flux, and a required key there is missing.  The deck reader does the same,
    checked against Apollo's own reader and eulerEqn plugin."""
    import numpy as np
    base = "<top>\n Equations = [eq]\n <eq>\n  Kind = eulerEqn\n  gas_gamma = 1.4\n{body} </eq>\n</top>\n"
    after = base.format(body="  <sub>\n   a = 1\n  </sub>\n  Numerical_Flux = HLL\n")
    before = base.format(body="  Numerical_Flux = HLL\n  <sub>\n   a = 1\n  </sub>\n")
    assert deck_equation(after)[2] == "LF"
    assert deck_equation(before)[2] == "HLL"
    with pytest.raises(Exception, match="gas_gamma"):
        deck_equation("<top>\n Equations = [eq]\n <eq>\n  Kind = eulerEqn\n  <sub>\n   a = 1\n  </sub>\n"
                      "  gas_gamma = 1.4\n </eq>\n</top>\n")
    orc = oracle_lib
    if not orc.RefPlugins.available():
        pytest.skip("Apollo's plugins are not built here")
    ref = orc.RefPlugins()
    qM, qP, n = np.array([1.0, 0.5, 0.2, 0.0, 2.5]), np.array([0.8, 0.1, -0.3, 0.0, 2.0]), np.array([0.6, 0.8])

    def flux(text):
        return ref.numflux(ref.lib.ref_eqn_create(text.encode()), n, qM.copy(), qP.copy())[0]
    np.testing.assert_array_equal(flux(after), flux(base.format(body="")))
    assert not np.array_equal(flux(before), flux(base.format(body="")))


def test_a_key_written_twice_takes_the_first_as_in_apollo(oracle_lib):
    """Of a key written twice in one block the first value counts, in the deck
    reader and in Apollo's own reader (checked through its eulerEqn flux)."""
    import numpy as np
    base = "<top>\n Equations = [eq]\n <eq>\n  Kind = eulerEqn\n{body} </eq>\n</top>\n"
    twice = base.format(body="  gas_gamma = 1.2\n  gas_gamma = 1.4\n")
    assert deck_equation(twice)[1][0] == 1.2
    orc = oracle_lib
    if not orc.RefPlugins.available():
        pytest.skip("Apollo's plugins are not built here")
    ref = orc.RefPlugins()
    qM, qP, n = np.array([1.0, 0.5, 0.2, 0.0, 2.5]), np.array([0.8, 0.1, -0.3, 0.0, 2.0]), np.array([0.6, 0.8])

    def flux(text):
        return ref.numflux(ref.lib.ref_eqn_create(text.encode()), n, qM.copy(), qP.copy())[0]
    np.testing.assert_array_equal(flux(twice), flux(base.format(body="  gas_gamma = 1.2\n")))
