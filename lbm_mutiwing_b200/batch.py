"""Many resident episodes advanced side by side on one GPU.

Every episode keeps its lattice, markers and geometry in HBM and owns its
CUDA streams; a pool of host threads (one per episode in flight) submits
the episodes' step segments (CUDA graphs), so the GPU overlaps the
latency-bound immersed-boundary chains and the bandwidth-bound bulk kernels
of different episodes.  The online server (``serve``) feeds the same
mechanism from client requests; ``advance_together`` is its offline form,
used to measure the batched throughput against serving the same episodes
one at a time.
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor
from typing import List, Sequence, Tuple

# more hardware work queues than the default 8 (read when the CUDA context is
# created): with many episodes' streams in flight, fewer queues would
# serialise independent work
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import api  # noqa: E402


def create(eps: Sequence, precision: int, device: int = 0, motion_source: int = api.MOTION_FILE,
           workers: int = 16) -> List[api.Simulation]:
    """Create the episodes (set-up runs on several host threads)."""
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda ep: api.Simulation(ep, precision, motion_source=motion_source, device=device), eps))


def advance_together(sims: Sequence[api.Simulation], steps: int, first_cycle: int = 1,
                     workers: int = 0) -> float:
    """Advance every episode by steps, all in flight at once; wall seconds."""
    n = len(sims)
    with ThreadPoolExecutor(max_workers=workers or n) as ex:
        t0 = time.perf_counter()
        list(ex.map(lambda s: s.step(steps, first_cycle=first_cycle, rows=False), sims))
        return time.perf_counter() - t0


def advance_one_at_a_time(eps: Sequence, steps: int, precision: int = api.PRECISION_FP64,
                          device: int = 0, warmup: int = 2) -> Tuple[float, int]:
    """Each episode alone (created, warmed up, timed, destroyed) in turn;
    returns (summed stepping seconds, node updates)."""
    total, nodes = 0.0, 0
    for ep in eps:
        with api.Simulation(ep, precision, device=device) as s:
            s.step(warmup, first_cycle=1, rows=False)
            t0 = time.perf_counter()
            s.step(steps, first_cycle=1 + warmup, rows=False)
            total += time.perf_counter() - t0
            nodes += ep.nx * ep.ny * steps
    return total, nodes
