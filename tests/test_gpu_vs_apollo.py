"""The B200 float64 right-hand side and stepper against results made by Apollo's
own code (tests/golden/apollo_rhs, written by tests/golden/make_apollo_rhs.py
with Apollo's WxNodalDG2dMethod compiled unmodified): every Euler flux with
the four Euler boundary conditions on elements listing their faces in every
order, the isentropic-vortex example, the Maxwell TM cavity, the cleaned
Maxwell form with both sources, advection, each of Apollo's Euler limiters
acting on the input; and for all but the Roe and Wave cases a few
SSPRK(5,2) steps taken through Apollo's right-hand side (the stage arithmetic
as PETSc's TSSSP documents it, the limiter rewriting each stage vector).  Agreement to 1e-12 relative L2
(1e-11 for the vortex, whose right-hand side is a small difference of O(1)
flux terms); no restatement stands between the CUDA kernels and Apollo's code.
"""
import pytest

from apollo_b200 import NodalDG2d
from golden_cases import APOLLO_NAMES, load_apollo, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", APOLLO_NAMES)
def test_rhs_matches_apollo(name):
    g = load_apollo(name)
    s = NodalDG2d(int(g["N"]), 0.5, g["equation"], tuple(g["eqp"]), g["mesh"], bcs=g["bcs"],
                  numerical_flux=g["numflux"], sources=g["sources"])
    if "limiter_kind" in g:  # Apollo's limiter in the method's Limiter list
        s.set_limiter(str(g["limiter_kind"]), tuple(g["limiter"]))
    got, sugg = s.step(float(g["t"]), float(g["dt"]), g["U"])
    assert rel_l2(got, g["rhs"]) <= (1e-11 if "vortex" in name else 1e-12)
    assert sugg == pytest.approx(float(g["sugg"]), rel=1e-13)
    if "steps" in g:  # SSPRK(5,2) steps with Apollo's dt policy through Apollo's right-hand side
        s.set_state(g["U"])
        t, dt = s.advance(int(g["steps"]), 0.0, float(g["dt"]))
        assert rel_l2(s.get_state(), g["U_end"]) <= 1e-12
        assert t == pytest.approx(float(g["t_end"]), rel=1e-13)
        assert dt == pytest.approx(float(g["dt_end"]), rel=1e-13)
