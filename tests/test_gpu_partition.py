"""Partitioned meshes on the GPU: P ranks (host threads on one device, each its
own handle and stream, traces exchanged through ThreadComm) compute bit for
bit what one handle on the whole mesh computes, in both precisions."""
import numpy as np
import pytest

from apollo_b200 import NodalDG2d, problems
from apollo_b200.distributed import DistNodalDG2d, partition
from thread_comm import run_ranks

pytestmark = pytest.mark.gpu

PROBLEMS = {
    "vortex_N4": lambda: problems.euler_vortex(n=21, N=4),
    "vortex_N2": lambda: problems.euler_vortex(n=17, N=2, beta=2.0),
    "tm_walls_N3": lambda: problems.maxwell_tm(n=17, N=3),
    "advection_N3": lambda: problems.advection(n=13, N=3),
}


def _whole(p, nsteps, precision):
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs)
    x, y = s.node_coords()
    s.set_state(np.ascontiguousarray(p.ic(x, y)))
    dt0 = s.init_dt()
    t, dt = s.advance(nsteps, 0.0, dt0, precision=precision)
    out = s.get_state(), t, dt, dt0, x
    s.close()
    return out


def _ranks(p, part, nsteps, precision):
    def fn(rank, comm):
        d = DistNodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, part, comm, bcs=p.bcs)
        x, y = d.node_coords()
        d.set_state(np.ascontiguousarray(p.ic(x, y)))
        dt0 = d.init_dt()
        t, dt = d.advance(nsteps, 0.0, dt0, precision=precision)
        U = d.get_state()
        d.close()
        return U, t, dt, dt0, x

    return run_ranks(int(part.max()) + 1, fn)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(PROBLEMS))
@pytest.mark.parametrize("P", [2, 3])
def test_partitioned_equals_whole(name, P, precision):
    p = PROBLEMS[name]()
    nsteps = 5
    Uw, tw, dtw, dt0w, xw = _whole(p, nsteps, precision)
    part = partition(p.mesh, P)
    res = _ranks(p, part, nsteps, precision)
    for r, (U, t, dt, dt0, x) in enumerate(res):
        ids = np.flatnonzero(part == r)
        np.testing.assert_array_equal(x, xw[ids])
        assert dt0 == dt0w
        # bit for bit: every face keeps its global orientation and the
        # reductions (MIN of dt, MAX of the wave speed) are exact
        np.testing.assert_array_equal(U, Uw[ids])
        assert t == tw and dt == dtw


def test_partitioned_many_ranks_and_continuation():
    """Six ranks on a periodic mesh; two calls of 3 steps equal one of 6."""
    p = PROBLEMS["vortex_N4"]()
    Uw, tw, dtw, _, _ = _whole(p, 6, "mixed")
    part = partition(p.mesh, 6)

    def fn(rank, comm):
        d = DistNodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, part, comm, bcs=p.bcs)
        x, y = d.node_coords()
        d.set_state(np.ascontiguousarray(p.ic(x, y)))
        dt0 = d.init_dt()
        t, dt = d.advance(3, 0.0, dt0, precision="mixed")
        t, dt = d.advance(3, t, dt, precision="mixed")
        U = d.get_state()
        d.close()
        return U, t, dt

    for r, (U, t, dt) in enumerate(run_ranks(6, fn)):
        np.testing.assert_array_equal(U, Uw[part == r])
        assert t == tw and dt == dtw


def test_partitioned_handle_refuses_whole_mesh_calls():
    from apollo_b200 import ApolloError
    p = PROBLEMS["vortex_N2"]()
    part = partition(p.mesh, 2)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, part=part, rank=1)
    x, y = s.node_coords()
    s.set_state(np.ascontiguousarray(p.ic(x, y)))
    with pytest.raises(ApolloError):
        s.advance(1, 0.0, 1e-3)
    with pytest.raises(ApolloError):
        s.step(0.0, 0.0, np.ascontiguousarray(p.ic(x, y)))
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_partitioned_hll_channel_equals_whole(precision):
    """Apollo's HLL flux (evaluated from both sides of a face, ghost slots
    included) and the channel's four boundary kinds on 2 ranks: bit for bit
    what one handle on the whole mesh computes."""
    from golden_cases import load
    g = load("euler_hll_N3")
    N, cfl, eq, eqp, bcs = int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["bcs"]
    s = NodalDG2d(N, cfl, eq, eqp, g["mesh"], bcs=bcs, numerical_flux="HLL")
    s.set_state(g["U0"])
    dt0 = s.init_dt()
    tw, dtw = s.advance(3, 0.0, dt0, precision=precision)
    Uw = s.get_state()
    s.close()
    part = partition(g["mesh"], 2)

    def fn(rank, comm):
        d = DistNodalDG2d(N, cfl, eq, eqp, g["mesh"], part, comm, bcs=bcs, numerical_flux="HLL")
        d.set_state(np.ascontiguousarray(g["U0"][part == rank]))
        t, dt = d.advance(3, 0.0, dt0, precision=precision)
        U = d.get_state()
        d.close()
        return U, t, dt

    for r, (U, t, dt) in enumerate(run_ranks(2, fn)):
        np.testing.assert_array_equal(U, Uw[part == r])
        assert t == tw and dt == dtw
