"""One process per GPU: rank plumbing for independent episodes.

Episodes never exchange data (each lattice, its wings and its force rows
belong to one episode), so N GPUs run N shards of episodes side by side with
no collective on the data path.  The only collectives are the timing ones: a
barrier around the timed region and a max over ranks of the elapsed time.
The backend is NCCL on GPUs and gloo on CPU (used by the tests).
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import List, Sequence, Tuple


def env() -> Tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0) -> Tuple[int, int, int]:
    """Join the process group when WORLD_SIZE > 1; returns env()."""
    rank, world, local = env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(local)
                kw["device_id"] = torch.device("cuda", local)
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def allmax(x: float) -> float:
    """Largest x over ranks (x itself with one rank)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


def shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Split episodes (by cost, e.g. nodes x steps) over ranks: longest first
    onto the least-loaded rank; every episode lands on exactly one rank and
    the result depends only on the costs (ties go to the lower rank)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def whole_job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Weak scaling: every rank processes units_per_rank; the job ends with the
    slowest rank."""
    return units_per_rank * world / seconds_max
