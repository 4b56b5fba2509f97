"""An in-process communicator for partitioned runs on one GPU: each rank is a
host thread with its own handle and stream; transfers are device copies made
after host barriers (every rank's stream synchronised first), so no kernel
ever waits on another rank's kernel."""
import threading

import torch


class ThreadGroup:
    def __init__(self, size: int):
        self.size = size
        self.barrier = threading.Barrier(size, timeout=120)
        self.slots = [None] * size


class ThreadComm:
    def __init__(self, group: ThreadGroup, rank: int):
        self.g = group
        self.rank = rank
        self.size = group.size

    @staticmethod
    def _sync():
        torch.cuda.current_stream().synchronize()

    def exchange(self, send, recv, peers, send_count, recv_count, block_bytes):
        self._sync()
        self.g.slots[self.rank] = (send, list(peers), list(send_count))
        self.g.barrier.wait()
        ro = 0
        for p, rc in zip(peers, recv_count):
            psend, ppeers, pcounts = self.g.slots[p]
            i = ppeers.index(self.rank)
            off = sum(pcounts[:i]) * block_bytes
            n = pcounts[i] * block_bytes
            assert n == rc * block_bytes
            recv[ro:ro + n].copy_(psend[off:off + n])
            ro += n
        self._sync()
        self.g.barrier.wait()

    def _gather(self, v):
        self.g.slots[self.rank] = v
        self.g.barrier.wait()
        vals = list(self.g.slots)
        self.g.barrier.wait()
        return vals

    def allreduce_max_(self, t):
        self._sync()
        m = max(self._gather(int(t.item())))
        t.fill_(m)

    def allreduce_min(self, x: float) -> float:
        return min(self._gather(float(x)))

    def allreduce_max_int(self, x: int) -> int:
        return max(self._gather(int(x)))


def run_ranks(size: int, fn):
    """fn(rank, comm) on `size` threads; returns the results, re-raising the first error."""
    group = ThreadGroup(size)
    out, errs = [None] * size, []

    def body(r):
        try:
            torch.cuda.set_device(0)
            out[r] = fn(r, ThreadComm(group, r))
        except BaseException as e:  # noqa: BLE001 - reported to the caller
            errs.append(e)
            group.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return out
