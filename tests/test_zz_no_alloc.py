"""The no-allocation float64 right-hand side (B200).

apollo_dg_rhs_noalloc serves callers that cannot allocate device memory at the
time they evaluate the right-hand side; its scratch lives in a static device
array.  It must give the same result as apollo_dg_rhs on device pointers, call
after call, and refuse meshes whose scratch exceeds the array.  This file is
named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from golden_cases import NAMES, load, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(s, t, dt, u, out, stream):
    sugg = C.c_double()
    rc = s.lib.apollo_dg_rhs_noalloc(s.h, t, dt, C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                                     C.byref(sugg), C.c_void_p(stream))
    return rc, sugg.value


@pytest.mark.parametrize("name", NAMES)
def test_noalloc_matches_rhs_twice(name):
    torch = pytest.importorskip("torch")
    g = load(name)
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"],
                  numerical_flux=g["numflux"], sources=g["sources"])
    u = torch.from_numpy(g["U0"]).cuda()
    if "limiter" in g:
        # the limiter needs scratch of its own: such handles are refused
        s.set_limiter(str(g.get("limiter_kind", "eulerLimiterHW")), g["limiter"])
        rc, _ = _noalloc(s, 0.25, 1e-3, u, torch.empty_like(u), torch.cuda.current_stream().cuda_stream)
        assert rc == 7
        return
    ref = torch.empty_like(u)
    _, sugg_ref = s.step(0.25, 1e-3, u, ref)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full_like(u, float("nan"))
        rc, sugg = _noalloc(s, 0.25, 1e-3, u, out, stream)
        torch.cuda.synchronize()
        assert rc == 0, (call, s.lib.apollo_dg_last_error(s.h))
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= TOL
        assert sugg == pytest.approx(sugg_ref, rel=1e-14)


def test_noalloc_second_input_after_first():
    """The array keeps the previous call's contents; a different input still gives its own result."""
    torch = pytest.importorskip("torch")
    g = load("euler_N4")
    s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=g["bcs"])
    stream = torch.cuda.current_stream().cuda_stream
    u1 = torch.from_numpy(g["U0"]).cuda()
    u2 = u1.clone()
    u2[..., 0] *= 1.01
    u2[..., 4] *= 1.02
    for u in (u1, u2, u1):
        ref = torch.empty_like(u)
        s.step(0.0, 0.0, u, ref)
        out = torch.empty_like(u)
        rc, _ = _noalloc(s, 0.0, 0.0, u, out, stream)
        torch.cuda.synchronize()
        assert rc == 0
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_noalloc_rejects_oversized_mesh():
    torch = pytest.importorskip("torch")
    p = problems.euler_vortex(n=130, N=4, fields=4)  # 33,282 elements: 80 MB of scratch
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    u = torch.zeros(s.shape, dtype=torch.float64, device="cuda")
    u[..., 0] = 1.0
    u[..., 3] = 2.5
    out = torch.empty_like(u)
    rc, _ = _noalloc(s, 0.0, 0.0, u, out, torch.cuda.current_stream().cuda_stream)
    assert rc == 8  # APOLLO_ERR_ARG
    assert b"64 MiB" in s.lib.apollo_dg_last_error(s.h)


def test_noalloc_refusals_say_why():
    """A handle without a mesh is refused with its reason in the error text."""
    torch = pytest.importorskip("torch")
    from apollo_b200.dg import _Config, load_library
    lib = load_library()
    cfg = _Config(3, 0.5, 0, None)
    h = C.c_void_p()
    assert lib.apollo_dg_create(C.byref(cfg), C.byref(h)) == 0
    try:
        u = torch.zeros(16, dtype=torch.float64, device="cuda")
        rc = lib.apollo_dg_rhs_noalloc(h, 0.0, 0.0, C.c_void_p(u.data_ptr()), C.c_void_p(u.data_ptr()), None,
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 7  # APOLLO_ERR_STATE
        assert b"no equation set" in lib.apollo_dg_last_error(h)
    finally:
        lib.apollo_dg_destroy(h)
