"""Float64 parity with the oracle on the benchmark configurations themselves
(B200): the stated meshes, orders and step counts rather than fixture-sized
grids.

* advection, N = 3, the jittered periodic 32 x 32 vertex grid (K = 1,922),
  200 steps of the adaptive SSPRK(5,2) stepper;
* the Euler vortex, N = 4, the jittered periodic 256 x 256 vertex grid
  (K = 130,050), 5 steps (the oracle takes about a second per step on 16
  threads);
* Maxwell TM with the mirror (PEC) boundary condition at N = 5 on a reduced
  48 x 48 vertex grid (K = 4,418), 60 steps, and on the configuration's own
  512 x 512 vertex grid (K = 522,242), 2 steps.

States after the steps agree with the oracle to 1e-12 relative L2, the time
reached and the next dt to 1e-13.  The mixed form is held against the float64
path on the same runs (1e-6 relative L2, the stated error of that form).
"""
import os

import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
MIXED_TOL = 1e-6


def _oracle(orc, p, eq, eqp, bcs=()):
    o = orc.Oracle(p.mesh, p.N, eq, eqp, bcs=bcs, cfl=p.cfl)
    o.set_threads(os.cpu_count() or 1)
    return o


def _run_both(s, o, U0_gpu, U0_cpu, steps):
    s.set_state(U0_gpu)
    dt0 = s.init_dt()
    dt0_cpu = o.init_dt(U0_cpu)
    assert dt0 == pytest.approx(dt0_cpu, rel=1e-14)
    t, dt = s.advance(steps, 0.0, dt0)
    U = s.get_state()
    Uc = U0_cpu.copy()
    n, tc, dtc = o.run(Uc, steps, 0.0, dt0_cpu)
    assert n == steps
    assert t == pytest.approx(tc, rel=1e-13)
    assert dt == pytest.approx(dtc, rel=1e-13)
    return U, Uc, dt0


def test_advection_config_full_size(oracle_lib):
    """Gaussian advected by (1, 0.5) on the periodic unit square, K = 1,922, N = 3, 200 steps."""
    orc = oracle_lib
    p = problems.advection(n=32, N=3)
    assert p.mesh.K == 1922
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    o = _oracle(orc, p, orc.EQ_ADVECTION, p.eq_params)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    U, Uc, dt0 = _run_both(s, o, U0, U0, 200)
    assert rel_l2(U, Uc) <= TOL
    # the mixed form on the same trajectory
    s.set_state(U0)
    s.advance(200, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= MIXED_TOL
    s.close()


def test_euler_vortex_config_mesh(oracle_lib):
    """The benchmark mesh itself: K = 130,050, N = 4, 5 steps against the oracle."""
    orc = oracle_lib
    p = problems.euler_vortex(n=256, N=4, fields=4)
    assert p.mesh.K == 130050
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    o = _oracle(orc, p, orc.EQ_EULER, p.eq_params)
    x, y = s.node_coords()
    U4 = np.ascontiguousarray(p.ic(x, y))
    U5 = np.zeros(U4.shape[:2] + (5,))
    U5[..., [0, 1, 2, 4]] = U4
    U, Uc, dt0 = _run_both(s, o, U4, U5, 5)
    assert np.all(Uc[..., 3] == 0.0)
    assert rel_l2(U, Uc[..., [0, 1, 2, 4]]) <= TOL
    s.set_state(U4)
    s.advance(5, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= MIXED_TOL
    s.close()


def test_maxwell_tm_config_order5_walls(oracle_lib):
    """Maxwell TM cavity mode with the mirror wall condition, N = 5, K = 4,418, 60 steps."""
    orc = oracle_lib
    p = problems.maxwell_tm(n=48, N=5)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    o = _oracle(orc, p, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),))
    x, y = s.node_coords()
    U3 = np.ascontiguousarray(p.ic(x, y))
    U8 = np.zeros(U3.shape[:2] + (8,))
    U8[..., 2:5] = U3
    U, Uc, dt0 = _run_both(s, o, U3, U8, 60)
    sel = [0, 1, 5, 6, 7]
    assert np.all(Uc[..., sel] == 0.0)
    assert rel_l2(U, Uc[..., 2:5]) <= TOL
    s.set_state(U3)
    s.advance(60, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= MIXED_TOL
    s.close()


def test_maxwell_tm_config_full_mesh(oracle_lib):
    """The Maxwell TM configuration's own mesh (512 x 512 vertices, K = 522,242),
    N = 5, mirror walls: 2 steps against the oracle (about 7 s per step on 16
    threads), the mixed form on the same steps."""
    orc = oracle_lib
    p = problems.maxwell_tm(n=512, N=5)
    assert p.mesh.K == 522242
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    o = _oracle(orc, p, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),))
    x, y = s.node_coords()
    U3 = np.ascontiguousarray(p.ic(x, y))
    U8 = np.zeros(U3.shape[:2] + (8,))
    U8[..., 2:5] = U3
    U, Uc, dt0 = _run_both(s, o, U3, U8, 2)
    assert rel_l2(U, Uc[..., 2:5]) <= TOL
    s.set_state(U3)
    s.advance(2, 0.0, dt0, precision="mixed")
    assert rel_l2(s.get_state(), U) <= MIXED_TOL
    s.close()
