"""Row-sharded solves over several ranks: the all-reduce the library calls for every exchange.

The library (db200_set_collective) splits one problem's n points into contiguous row blocks (db200_row_shard): each
rank computes its rows of Y = K Omega with no exchange, and all-reduces the l x l Grams of CholeskyQR2 and of the
Nystrom core, the gathered Q of the power and final passes (a sum of zero-filled row blocks), and per Newton step the
r x r capacity matrix, the r-vectors Z^T x and the scalar sums, maxima and minima.  This module supplies that
all-reduce:

  * TorchCollective: torch.distributed (NCCL for device buffers, one process per GPU; gloo for host buffers), the
    production plumbing, replacing the MPI Allreduce / Allgatherv of the reference's distributed matrices
    (include/darray.h:737-1054, include/lapack_like.h:308);
  * LoopbackCollective: `world` ranks as threads of one process, each with its own context and stream, reduced on
    the host side of the threads' rendezvous (every rank's stream is synchronised before the exchange, so no kernel
    ever waits on another rank's kernel): the in-process check of the sharded path on one device.

Usage, one process per GPU (torchrun):

    ctx = Context(local_rank, torch.cuda.current_stream().cuda_stream)
    coll = TorchCollective()            # default process group
    coll.attach(ctx)
    start, count = row_shard(n, world, rank)
    ctx.svm_solve(n, d, l, q, X, d, y, Om, n, gamma, C, a_rows, Z_rows, count)   # this rank's rows of a and Z
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib

SUM, MAX, MIN = _lib.REDUCE_SUM, _lib.REDUCE_MAX, _lib.REDUCE_MIN


def row_shard(n: int, world: int, rank: int) -> tuple[int, int]:
    """(start, count) of rank's contiguous row block (db200_row_shard)."""
    s, c = ctypes.c_int(), ctypes.c_int()
    st = _lib.load().db200_row_shard(n, world, rank, ctypes.byref(s), ctypes.byref(c))
    if st != 0:
        raise _lib.DB200Error(st, f"row_shard(n={n}, world={world}, rank={rank})")
    return s.value, c.value


class _DeviceBuffer:
    """A device FP64 buffer seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def view(ptr: int, count: int, device: str):
    """torch tensor over count FP64 values at ptr (device "cuda": device memory, "cpu": host memory)."""
    import torch
    if device == "cpu":
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=(count,))
        return torch.from_numpy(arr)
    return torch.as_tensor(_DeviceBuffer(ptr, count), device="cuda")


def _sync_stream(stream: int | None, device: str):
    if device == "cpu":
        return
    import torch
    if stream:
        torch.cuda.ExternalStream(stream).synchronize()
    else:
        torch.cuda.synchronize()


class _Callback:
    """Common part: the ctypes callback, with the first failure kept for the caller's report."""

    def __init__(self):
        self.error: BaseException | None = None
        self.calls = 0
        self.values = 0
        self.fn = _lib.ALLREDUCE_FN(self._entry)

    def _entry(self, user, buf, count, op, stream):
        try:
            self.calls += 1
            self.values += int(count)
            self.reduce(int(buf), int(count), int(op), stream)
            return 0
        except BaseException as e:  # reported to the library as a failed collective
            if self.error is None:
                self.error = e
            return 1


class TorchCollective(_Callback):
    """All-reduce over a torch.distributed process group (None: the default group).  device "cuda" for the
    library's device buffers (NCCL), "cpu" for host buffers (gloo)."""

    def __init__(self, group=None, device: str = "cuda"):
        super().__init__()
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = device
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.ops = {SUM: dist.ReduceOp.SUM, MAX: dist.ReduceOp.MAX, MIN: dist.ReduceOp.MIN}

    def reduce(self, buf: int, count: int, op: int, stream):
        import torch
        _sync_stream(stream, self.device)  # the buffer is ready on the library's stream
        t = view(buf, count, self.device)
        self.dist.all_reduce(t, op=self.ops[op], group=self.group)
        if self.device != "cpu":
            torch.cuda.current_stream().synchronize()  # the result is in place before the library goes on

    def attach(self, ctx):
        ctx.set_collective(self.world, self.rank, self.fn)


class LoopbackCollective:
    """`world` ranks as threads of one process.  rank(k) is rank k's callback; every rank calls it with the same
    count and op in the same order.  Rank 0's thread combines the buffers once all ranks have arrived and every
    rank's stream has been synchronised; a rendezvous that does not complete within `timeout` seconds fails the
    call on every rank (the library then returns DB200_ERR_COLLECTIVE)."""

    def __init__(self, world: int, device: str = "cuda", timeout: float = 120.0):
        self.world = world
        self.device = device
        self.barrier = threading.Barrier(world, timeout=timeout)
        self.slots: list = [None] * world
        self.failed = False
        self.ranks = [self._Rank(self, k) for k in range(world)]

    class _Rank(_Callback):
        def __init__(self, parent, k):
            super().__init__()
            self.parent, self.k = parent, k

        def reduce(self, buf, count, op, stream):
            p = self.parent
            _sync_stream(stream, p.device)
            p.slots[self.k] = (buf, count, op)
            p.barrier.wait()
            if self.k == 0:
                try:
                    p.failed = False
                    if len({(c, o) for _, c, o in p.slots}) != 1:
                        raise RuntimeError(f"ranks disagree on the collective: {[(c, o) for _, c, o in p.slots]}")
                    ts = [view(b, c, p.device) for b, c, _ in p.slots]
                    import torch
                    stacked = torch.stack(ts)
                    res = {SUM: lambda x: x.sum(0), MAX: lambda x: x.amax(0), MIN: lambda x: x.amin(0)}[op](stacked)
                    for t in ts:
                        t.copy_(res)
                    if p.device != "cpu":
                        torch.cuda.synchronize()
                except BaseException:
                    p.failed = True
                    raise
                finally:
                    p.barrier.wait()
            else:
                p.barrier.wait()
                if p.failed:
                    raise RuntimeError("rank 0 could not combine the buffers")

    def rank(self, k: int) -> _Callback:
        return self.ranks[k]

    def attach(self, ctx, k: int):
        ctx.set_collective(self.world, k, self.ranks[k].fn)
