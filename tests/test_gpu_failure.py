"""Failure paths (B200), none of which faults, traps or hangs the GPU.

* A bounded device wait of the mixed-precision stage kernel runs out: a test
  switch points the kernel's first wait at a barrier that nothing completes,
  with a short poll limit.  The kernel drains, frees its tensor memory and
  returns; the call reports APOLLO_ERR_TIMEOUT, and once the switch is
  cleared the same handle computes exactly what it computed before.
* Host-side injections (Apollo calls exit(1) in these places): a clockwise and
  a degenerate element (APOLLO_ERR_MESH), and a device allocation that fails
  part way through a mesh set-up (APOLLO_ERR_ALLOC), after which the handle
  holds no mesh and accepts the next one.
"""
import ctypes as C

import numpy as np
import pytest

from apollo_b200 import ApolloError, NodalDG2d, problems

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
ERR_MESH, ERR_TIMEOUT, ERR_ALLOC = 2, 5, 9


def _vortex(n=12, N=4):
    p = problems.euler_vortex(n=n, N=N, fields=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    return p, s, np.ascontiguousarray(p.ic(x, y))


def _set_mesh(s, m):
    return s.lib.apollo_dg_set_mesh(s.h, m.nverts, m.vx.ctypes.data_as(_dp), m.vy.ctypes.data_as(_dp), m.K,
                                    m.etov.ctypes.data_as(_ip), m.face_tag.ctypes.data_as(_ip),
                                    m.vert_canon.ctypes.data_as(_ip))


def test_mixed_stage_wait_timeout_and_recovery():
    p, s, U0 = _vortex()
    ref, _ = s.step(0.0, 0.0, U0, precision="mixed")
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 2000, 1))
    with pytest.raises(ApolloError) as e:
        s.step(0.0, 0.0, U0, precision="mixed")
    assert e.value.code == ERR_TIMEOUT
    assert "timed out" in str(e.value)
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 0, 0))
    again, _ = s.step(0.0, 0.0, U0, precision="mixed")
    np.testing.assert_array_equal(again, ref)
    # whole mixed steps on the recovered handle equal those of a fresh handle
    s.set_state(U0)
    dt = s.init_dt()
    s.advance(2, 0.0, dt, precision="mixed")
    fresh = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    fresh.set_state(U0)
    fresh.advance(2, 0.0, dt, precision="mixed")
    np.testing.assert_array_equal(s.get_state(), fresh.get_state())
    # a short poll limit alone (no stall) does not disturb a normal launch
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 1 << 16, 0))
    np.testing.assert_array_equal(s.step(0.0, 0.0, U0, precision="mixed")[0], ref)
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 0, 0))


def test_timeout_inside_a_step_is_reported():
    p, s, U0 = _vortex()
    s.set_state(U0)
    dt = s.init_dt()
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 2000, 1))
    with pytest.raises(ApolloError) as e:
        s.advance(1, 0.0, dt, precision="mixed")
    assert e.value.code == ERR_TIMEOUT
    s._check(s.lib.apollo_dg_debug_set_waits(s.h, 0, 0))
    s.set_state(U0)
    s.advance(1, 0.0, dt, precision="mixed")
    assert np.all(np.isfinite(s.get_state()))


@pytest.mark.parametrize("defect", ["clockwise", "degenerate"])
def test_bad_element_is_refused(defect):
    p, s, U0 = _vortex(n=9)
    m = problems.euler_vortex(n=9, N=4, fields=4).mesh
    if defect == "clockwise":
        m.etov[5, [1, 2]] = m.etov[5, [2, 1]]
    else:
        # vertex 2 of element 5 moved onto the midpoint of its edge (v0, v1)
        a, b, c = m.etov[5]
        m.vx[c] = 0.5 * (m.vx[a] + m.vx[b])
        m.vy[c] = 0.5 * (m.vy[a] + m.vy[b])
    assert _set_mesh(s, m) == ERR_MESH
    assert "element" in s.lib.apollo_dg_last_error(s.h).decode()
    assert s.lib.apollo_dg_num_elements(s.h) == 0
    with pytest.raises(ApolloError):
        s.step(0.0, 0.0, U0)
    # the handle takes a good mesh afterwards
    assert _set_mesh(s, p.mesh) == 0
    out, _ = s.step(0.0, 0.0, U0)
    ref, _ = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh).step(0.0, 0.0, U0)
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("nth", [0, 12, 20])
def test_failed_allocation_leaves_no_mesh(nth):
    """nth device allocation of the mesh set-up fails: operator uploads (0),
    state buffers (12), the mixed form's trace buffers (20, after the element
    count is known)."""
    p, s, U0 = _vortex(n=9)
    ref, _ = s.step(0.0, 0.0, U0)
    ref_m, _ = s.step(0.0, 0.0, U0, precision="mixed")
    s.lib.apollo_dg_debug_fail_alloc(nth)
    try:
        rc = _set_mesh(s, p.mesh)
    finally:
        s.lib.apollo_dg_debug_fail_alloc(-1)
    assert rc == ERR_ALLOC
    assert "out of memory" in s.lib.apollo_dg_last_error(s.h).decode()
    assert s.lib.apollo_dg_num_elements(s.h) == 0
    with pytest.raises(ApolloError):
        s.step(0.0, 0.0, U0)
    assert _set_mesh(s, p.mesh) == 0
    np.testing.assert_array_equal(s.step(0.0, 0.0, U0)[0], ref)
    np.testing.assert_array_equal(s.step(0.0, 0.0, U0, precision="mixed")[0], ref_m)
