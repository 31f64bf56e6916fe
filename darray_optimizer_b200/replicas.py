"""One process per GPU, independent replicas of the hot path (the path has no exchange step).

The collectives here are timing plumbing only: a barrier before and after the timed region and the max of the
per-rank times.  NCCL on GPUs; the same code runs on CPU with gloo (tests use world size 2).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Replicas:
    world: int
    rank: int
    local: int
    backend: str | None


def init(backend: str | None = None, timeout_s: int = 120) -> Replicas:
    """Read RANK / LOCAL_RANK / WORLD_SIZE from the launcher's environment and join the process group when
    WORLD_SIZE > 1 (nccl with a device id when CUDA is available, else gloo)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return Replicas(world, rank, local, backend if world > 1 else None)


def barrier(r: Replicas) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()


def all_max(r: Replicas, x: float) -> float:
    """Max over ranks (the whole job's time is the slowest replica's)."""
    if r.world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if r.backend == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_throughput(r: Replicas, work_per_rank: float, seconds_this_rank: float) -> float:
    """Aggregate throughput of N replicas: all ranks' work over the slowest rank's time (weak scaling)."""
    return r.world * work_per_rank / all_max(r, seconds_this_rank)


def finalize(r: Replicas) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
