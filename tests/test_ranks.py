"""Rank plumbing of the multi-GPU path on CPU: two gloo ranks, each with its
own shard of independent episodes and its own elapsed time; the whole-job
rate uses the slowest rank.  No data-path collective exists to test."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lbm_mutiwing_b200 import ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, _ = ranks.init("gloo", timeout_s=60)
    costs = [float(c) for c in (5, 1, 4, 4, 2, 8, 3)]
    mine = ranks.shard(costs, w)[r]
    elapsed = 1.0 + r                      # rank 1 is the slow one
    ranks.barrier()
    m = ranks.allmax(elapsed)
    out.put((r, mine, m, ranks.whole_job_rate(100.0, w, m)))
    ranks.finish()


def test_two_gloo_ranks_max_time_and_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, m0, v0), (r1, s1, m1, v1) = res
    assert m0 == m1 == 2.0
    assert v0 == v1 == 100.0
    assert sorted(s0 + s1) == list(range(7)) and not set(s0) & set(s1)


def test_shard_is_balanced_and_deterministic():
    costs = [10, 9, 8, 7, 6, 5, 4, 3, 2, 1]
    a = ranks.shard(costs, 3)
    assert a == ranks.shard(costs, 3)
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) - min(loads) <= max(costs)
    assert ranks.shard(costs, 1) == [list(range(10))]


def test_single_rank_needs_no_process_group():
    assert ranks.allmax(3.5) == 3.5
    ranks.barrier()
    assert ranks.whole_job_rate(10.0, 1, 2.0) == 5.0
