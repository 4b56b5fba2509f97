"""Partitioned meshes: one rank per GPU, cut-face traces exchanged once per stage.

Apollo distributes its mesh with PETSc DMPlex (overlap 1) and refreshes the
ghost cells with ``DMGlobalToLocal`` before each right-hand side, then reduces
the dt estimate with ``MPI_Allreduce`` (src/solvers/apsolver.cc:318-392,
431-433).  Here each rank holds its elements plus ghost slots for the face
traces of remote neighbours (``apollo_dg_set_mesh_partition``); per stage the
library packs the traces of the cut faces into a send buffer, the
communicator moves them (NCCL point-to-point through ``torch.distributed`` on
GPUs, gloo on CPU), and the library unpacks them into the ghost slots before
the face fluxes.  The ranks together compute bit for bit what one handle on
the whole mesh computes.

``comm`` objects provide ``rank``, ``size``, ``exchange``, ``allreduce_max_``
(in place, int64 tensor), ``allreduce_min`` and ``allreduce_max_int`` (host
scalars); ``TorchComm`` is the ``torch.distributed`` one.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .dg import PREC, ApolloError, HaloSizes, NodalDG2d, _dp, _ip, load_library
from .mesh import Mesh


def partition(mesh: Mesh, nparts: int) -> np.ndarray:
    """Recursive coordinate bisection of the element centroids (apollo_dg_partition)."""
    lib = load_library()
    part = np.empty(mesh.K, dtype=np.int32)
    code = lib.apollo_dg_partition(mesh.nverts, mesh.vx.ctypes.data_as(_dp), mesh.vy.ctypes.data_as(_dp), mesh.K,
                                   mesh.etov.ctypes.data_as(_ip), nparts, part.ctypes.data_as(_ip))
    if code:
        raise ApolloError(code, f"partition of {mesh.K} elements into {nparts} parts")
    return part


@dataclass
class HaloPlan:
    local: np.ndarray       # global ids of the rank's elements
    ghost: np.ndarray       # global ids of the remote neighbours
    peers: list
    send_count: list
    recv_count: list
    send_faces: np.ndarray  # global face id 3k+f of the local side, per block sent
    recv_faces: np.ndarray  # global face id of the remote side, per block received


def halo_plan(mesh: Mesh, part: np.ndarray, rank: int) -> HaloPlan:
    """The rank's halo plan (apollo_dg_halo_plan); host only."""
    lib = load_library()
    part = np.ascontiguousarray(part, dtype=np.int32)
    sz = HaloSizes()
    args = (mesh.nverts, mesh.K, mesh.etov.ctypes.data_as(_ip), mesh.face_tag.ctypes.data_as(_ip),
            mesh.vert_canon.ctypes.data_as(_ip), part.ctypes.data_as(_ip), rank, C.byref(sz))
    code = lib.apollo_dg_halo_plan(*args, None, None, None, None, None, None, None)
    if code:
        raise ApolloError(code, "halo plan")
    arr = [np.zeros(n, dtype=np.int32) for n in (sz.n_local, sz.n_ghost, sz.n_peers, sz.n_peers, sz.n_peers,
                                                  sz.n_send, sz.n_recv)]
    code = lib.apollo_dg_halo_plan(*args, *[a.ctypes.data_as(_ip) for a in arr])
    if code:
        raise ApolloError(code, "halo plan")
    return HaloPlan(arr[0], arr[1], arr[2].tolist(), arr[3].tolist(), arr[4].tolist(), arr[5], arr[6])


class TorchComm:
    """Exchange and reductions over a ``torch.distributed`` process group
    (NCCL for CUDA buffers, gloo for CPU ones); the group ranks are the
    partition's part ids."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def exchange(self, send, recv, peers, send_count, recv_count, block_bytes):
        """Blocks for each peer, back to back in peer order: send -> peer, peer -> recv."""
        dist = self.dist
        ops, so, ro = [], 0, 0
        for p, sc, rc in zip(peers, send_count, recv_count):
            if sc:
                ops.append(dist.P2POp(dist.isend, send[so:so + sc * block_bytes], self._global(p), self.group))
            if rc:
                ops.append(dist.P2POp(dist.irecv, recv[ro:ro + rc * block_bytes], self._global(p), self.group))
            so += sc * block_bytes
            ro += rc * block_bytes
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce_max_(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def _host_reduce(self, x, op, dtype):
        import torch
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([x], dtype=dtype, device=dev)
        self.dist.all_reduce(t, op=op, group=self.group)
        return t.item()

    def allreduce_min(self, x: float) -> float:
        import torch
        return float(self._host_reduce(x, self.dist.ReduceOp.MIN, torch.float64))

    def allreduce_max_int(self, x: int) -> int:
        import torch
        return int(self._host_reduce(x, self.dist.ReduceOp.MAX, torch.int64))


class DistNodalDG2d:
    """One rank's share of a partitioned nodal-DG discretisation and its
    SSPRK(5,2) stepper (Apollo's dt policy, dt reduced over the ranks)."""

    def __init__(self, N: int, cfl: float, equation: str, eq_params, mesh: Mesh, part, comm, bcs=(),
                 device: int = 0, numerical_flux: str = "LF"):
        import torch
        self.comm = comm
        self.torch_stream = torch.cuda.Stream(device=device)
        self.solver = NodalDG2d(N, cfl, equation, eq_params, mesh, bcs=bcs, device=device,
                                stream=self.torch_stream.cuda_stream, part=part, rank=comm.rank,
                                numerical_flux=numerical_flux)
        s = self.solver
        self.lib, self.h = s.lib, s.h
        n = C.c_int()
        s._check(self.lib.apollo_dg_halo_info(self.h, PREC["fp64"], C.byref(n), None, None, None, None))
        peers, sc, rc = (np.zeros(n.value, dtype=np.int32) for _ in range(3))
        blk = {}
        for prec in ("fp64", "mixed"):
            b = C.c_int(0)
            code = self.lib.apollo_dg_halo_info(self.h, PREC[prec], None, peers.ctypes.data_as(_ip),
                                                sc.ctypes.data_as(_ip), rc.ctypes.data_as(_ip), C.byref(b))
            if code == 0:
                blk[prec] = b.value
        self.peers, self.send_count, self.recv_count = peers.tolist(), sc.tolist(), rc.tolist()
        self.block_bytes = blk
        big = blk["fp64"]
        dev = torch.device("cuda", device)
        self.send = torch.zeros(max(1, sum(self.send_count)) * big, dtype=torch.uint8, device=dev)
        self.recv = torch.zeros(max(1, sum(self.recv_count)) * big, dtype=torch.uint8, device=dev)
        self.lam = torch.zeros(2, dtype=torch.int64, device=dev)  # word 0 is reduced; 16 bytes keep alignment
        s._check(self.lib.apollo_dg_halo_bind(self.h, self.send.data_ptr(), self.send.numel(), self.recv.data_ptr(),
                                              self.recv.numel(), self.lam.data_ptr()))
        torch.cuda.synchronize(dev)  # the buffers' fills (torch's stream) before the library's stream uses them

    @property
    def shape(self):
        return self.solver.shape

    def node_coords(self):
        return self.solver.node_coords()

    def set_state(self, U):
        self.solver.set_state(U)

    def get_state(self, out=None):
        return self.solver.get_state(out)

    def init_dt(self) -> float:
        """Apollo's initial dt over the whole mesh: the MIN over ranks of the local estimates."""
        return self.comm.allreduce_min(self.solver.init_dt())

    def advance(self, nsteps: int, t: float, dt: float, precision: str = "fp64"):
        """nsteps steps of every rank from (t, dt); returns (t, dt for the next step)."""
        import torch
        lib, h, p = self.lib, self.h, PREC[precision]
        blk = self.block_bytes[precision]
        chk = self.solver._check
        chk(lib.apollo_dg_dist_start(h, t, dt, p))
        with torch.cuda.stream(self.torch_stream):
            lam = self.lam[:1]
            for _ in range(nsteps):
                for stage in range(5):
                    chk(lib.apollo_dg_stage_begin(h, stage, p))
                    self.comm.exchange(self.send, self.recv, self.peers, self.send_count, self.recv_count, blk)
                    chk(lib.apollo_dg_stage_end(h, stage, p))
                self.comm.allreduce_max_(lam)
                chk(lib.apollo_dg_step_end(h))
        tt, dd, code = C.c_double(), C.c_double(), 0
        code = lib.apollo_dg_get_time(h, C.byref(tt), C.byref(dd))
        # every rank fails together: a rank's error ends the others' calls too
        worst = self.comm.allreduce_max_int(code)
        if code:
            chk(code)
        if worst:
            raise ApolloError(worst, "another rank failed")
        return tt.value, dd.value

    def close(self):
        self.solver.close()
