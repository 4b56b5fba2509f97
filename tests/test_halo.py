"""Partitioned meshes on the CPU: partitions, halo plans against the oracle's
own face pairing, and the per-stage trace exchange through torch.distributed
(gloo, 2 and 3 ranks) with blocks laid out as the library packs them."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from apollo_b200 import ApolloError, problems
from apollo_b200.distributed import TorchComm, halo_plan, partition

# (problem, oracle equation code, equation parameters, oracle boundary conditions)
CASES = {
    "vortex": (lambda: problems.euler_vortex(n=17, N=3, fields=5), 1, (1.4, 0.0, 0.0), ()),
    "tm_walls": (lambda: problems.maxwell_tm(n=13, N=2, fields=8), 2, (1.0, 0.0, 0.0), ((2, ()),)),
}


def _oracle(orc, name):
    mk, eq, eqp, bcs = CASES[name]
    p = mk()
    return p, orc.Oracle(p.mesh, p.N, eq, eqp, bcs=bcs, cfl=p.cfl)


def _cuts(conn, part):
    """Cut faces from the oracle's connectivity: (k, f, partner element, partner face)."""
    out = []
    K = conn.shape[0]
    for k in range(K):
        for f in range(3):
            nb = conn[k, 2 * f]
            if nb >= 0 and part[nb] != part[k]:
                out.append((k, f, nb, conn[k, 2 * f + 1]))
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_partition_balanced_and_deterministic(name):
    m = CASES[name][0]().mesh
    for P in (1, 2, 3, 5, 8):
        a, b = partition(m, P), partition(m, P)
        np.testing.assert_array_equal(a, b)
        counts = np.bincount(a, minlength=P)
        assert counts.min() >= 1 and counts.max() - counts.min() <= 1
        assert a.min() == 0 and a.max() == P - 1


def test_partition_rejects_bad_counts():
    m = CASES["vortex"][0]().mesh
    with pytest.raises(ApolloError):
        partition(m, 0)
    with pytest.raises(ApolloError):
        partition(m, m.K + 1)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("P", [2, 3, 4, 6])
def test_halo_plans_match_oracle_pairing(oracle_lib, name, P):
    p, o = _oracle(oracle_lib, name)
    m = p.mesh
    part = partition(m, P)
    plans = [halo_plan(m, part, r) for r in range(P)]
    np.testing.assert_array_equal(np.sort(np.concatenate([pl.local for pl in plans])), np.arange(m.K))
    cuts = _cuts(o.connectivity(), part)
    for r, pl in enumerate(plans):
        np.testing.assert_array_equal(pl.local, np.flatnonzero(part == r))
        mine = [c for c in cuts if part[c[0]] == r]
        assert sorted(pl.ghost.tolist()) == sorted({c[2] for c in mine})
        assert pl.peers == sorted({int(part[c[2]]) for c in mine})
        so = ro = 0
        for s, sc, rc in zip(pl.peers, pl.send_count, pl.recv_count):
            sent = sorted(3 * c[0] + c[1] for c in mine if part[c[2]] == s)
            recvd = sorted(3 * c[2] + c[3] for c in mine if part[c[2]] == s)
            assert pl.send_faces[so:so + sc].tolist() == sent
            assert pl.recv_faces[ro:ro + rc].tolist() == recvd
            # the peer's plan names the same blocks in the same order
            q = plans[s]
            i = q.peers.index(r)
            q0 = sum(q.send_count[:i])
            assert q.send_faces[q0:q0 + q.send_count[i]].tolist() == recvd
            so += sc
            ro += rc


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port, name):
    import torch
    import torch.distributed as dist
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        p, o = _oracle(orc, name)
        m = p.mesh
        part = partition(m, world)
        plan = halo_plan(m, part, rank)
        x, y = o.node_coords()
        U = np.ascontiguousarray(p.ic(x, y))
        I = o.operator(3)  # [3 Ng][Np]: nodes to the face Gauss points, own order
        Ng, M = o.Ng, o.meqn

        def trace(k, f):
            return I[f * Ng:(f + 1) * Ng] @ U[k]

        # pack this rank's blocks from its own elements only, as the library does
        send = torch.zeros(max(1, len(plan.send_faces)) * Ng * M, dtype=torch.float64)
        sv = send.numpy().reshape(-1, Ng, M)
        for j, gf in enumerate(plan.send_faces):
            assert part[gf // 3] == rank
            sv[j] = trace(gf // 3, gf % 3)
        recv = torch.full((max(1, len(plan.recv_faces)) * Ng * M,), np.nan, dtype=torch.float64)
        comm = TorchComm()
        assert (comm.rank, comm.size) == (rank, world)
        comm.exchange(send.view(torch.uint8), recv.view(torch.uint8), plan.peers, plan.send_count, plan.recv_count,
                      Ng * M * 8)
        rv = recv.numpy().reshape(-1, Ng, M)
        conn = o.connectivity()
        for j, gf in enumerate(plan.recv_faces):
            kr, fr = divmod(int(gf), 3)
            assert part[kr] != rank
            assert part[conn[kr, 2 * fr]] == rank  # the oracle pairs it with one of ours
            np.testing.assert_array_equal(rv[j], trace(kr, fr))
        # dt reductions: MIN of the local estimates, MAX of the wave-speed bits
        assert comm.allreduce_min(0.5 + rank) == 0.5
        assert comm.allreduce_max_int(rank) == world - 1
        speeds = np.array([0.75, 2.5, 1.125, 3.0625])[:world]
        lam = torch.from_numpy(np.array([speeds[rank]]).view(np.int64).copy())
        comm.allreduce_max_(lam)
        assert lam.numpy().view(np.float64)[0] == speeds.max()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_trace_exchange_gloo(oracle_lib, name, world):
    import torch.multiprocessing as mp
    mp.spawn(_exchange_worker, args=(world, _free_port(), name), nprocs=world, join=True)
