"""Asynchronous state copies and steps (apollo_dg_set_state_async,
apollo_dg_get_state_async, apollo_dg_step_async): queued on the handle's
stream without host waits, they give what the synchronous calls give."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems

pytestmark = pytest.mark.gpu


def _handle(p, stream=None):
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, stream=stream)
    x, y = s.node_coords()
    return s, np.ascontiguousarray(p.ic(x, y))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_copies_match_synchronous_calls(precision):
    import torch
    p = problems.euler_vortex(n=17, N=4)
    s, U0 = _handle(p)
    s.set_state(U0)
    dt0 = s.init_dt()
    t, dt = s.advance(2, 0.0, dt0, precision=precision)
    ref = s.get_state()

    # device tensors in and out
    dU = torch.from_numpy(U0).cuda()
    dO = torch.empty_like(dU)
    torch.cuda.synchronize()
    s.set_state_async(dU)
    s.advance_async(2, 0.0, dt0, precision=precision)
    s.get_state_async(dO)
    s.synchronize()
    np.testing.assert_array_equal(dO.cpu().numpy(), ref)
    assert s.time() == (t, dt)

    # page-locked host memory in and out
    hU = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
    hU.numpy()[...] = U0
    hO = torch.zeros(s.shape, dtype=torch.float64, pin_memory=True)
    s.set_state_async(hU)
    s.advance_async(2, 0.0, dt0, precision=precision)
    s.get_state_async(hO)
    s.synchronize()
    np.testing.assert_array_equal(hO.numpy(), ref)
    s.close()


def test_back_to_back_async_steps_keep_their_own_times():
    """Each apollo_dg_step_async call carries its own (t, dt) to the device:
    calls queued without a host wait in between do not see each other's."""
    import torch
    p = problems.euler_vortex(n=13, N=3)
    s, U0 = _handle(p)
    s.set_state(U0)
    dt0 = s.init_dt()
    expect = []
    for k in range(4):
        s.set_state(U0)
        t, dt = s.advance(1, 0.1 * k, dt0 * (1.0 - 0.1 * k), precision="fp64")
        expect.append((s.get_state(), t, dt))
    outs = [torch.empty(s.shape, dtype=torch.float64, device="cuda") for _ in range(4)]
    dU = torch.from_numpy(U0).cuda()
    torch.cuda.synchronize()
    for k in range(4):
        s.set_state_async(dU)
        s.advance_async(1, 0.1 * k, dt0 * (1.0 - 0.1 * k), precision="fp64")
        s.get_state_async(outs[k])
    s.synchronize()
    for k in range(4):
        np.testing.assert_array_equal(outs[k].cpu().numpy(), expect[k][0])
    assert s.time() == expect[-1][1:]
    s.close()


def test_streamed_steps_on_a_caller_stream():
    """The bench's streamed pattern: uploads and downloads on their own streams,
    the handle on a caller stream, ordered by events only."""
    import torch
    p = problems.euler_vortex(n=17, N=4)
    cs = torch.cuda.Stream()
    s, U0 = _handle(p, stream=cs.cuda_stream)
    s.set_state(U0)
    dt0 = s.init_dt()
    s.advance(1, 0.0, dt0, precision="mixed")
    ref = s.get_state()
    n = 6
    hU = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
    hU.numpy()[...] = U0
    hO = [torch.zeros(s.shape, dtype=torch.float64, pin_memory=True) for _ in range(n)]
    dU = [torch.empty(s.shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    dO = [torch.empty(s.shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_up, ev_taken, ev_out, ev_down = ([torch.cuda.Event() for _ in range(2)] for _ in range(4))
    torch.cuda.synchronize()
    for b in range(2):
        ev_taken[b].record(cs)
        ev_down[b].record(down)
    for i in range(n):
        b = i % 2
        up.wait_event(ev_taken[b])
        with torch.cuda.stream(up):
            dU[b].copy_(hU, non_blocking=True)
            ev_up[b].record(up)
        cs.wait_event(ev_up[b])
        s.set_state_async(dU[b])
        ev_taken[b].record(cs)
        s.advance_async(1, 0.0, dt0, precision="mixed")
        cs.wait_event(ev_down[b])
        s.get_state_async(dO[b])
        ev_out[b].record(cs)
        down.wait_event(ev_out[b])
        with torch.cuda.stream(down):
            hO[i].copy_(dO[b], non_blocking=True)
            ev_down[b].record(down)
    torch.cuda.synchronize()
    for i in range(n):
        np.testing.assert_array_equal(hO[i].numpy(), ref)
    s.close()
