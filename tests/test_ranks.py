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


class _FakeEngine:
    """Stands in for the packed GPU engine: 'episodes' are names, advancing
    records (episode, first cycle, steps) and takes a time proportional to
    the node updates of the call."""

    def __init__(self, log):
        self.log = log

    def create(self, eps):
        return [e.name for e in eps]

    def advance(self, sims, steps, first_cycle):
        for s in sims:
            self.log.append((s, first_cycle, steps))
        return 1e-9 * steps * len(sims)

    def close(self, sims):
        self.log.append(("closed", len(sims)))


def _batch_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from lbm_mutiwing_b200 import batch, workloads as wl
    r, w, _ = ranks.init("gloo", timeout_s=60)
    eps = wl.mixed_batch(16, steps=4)
    log = []
    mine, nu, sec = batch.sharded_packed_run(eps, 10, 3, r, w, engine=_FakeEngine(log), barrier=ranks.barrier)
    smax = ranks.allmax(sec)
    out.put((r, mine, nu, smax, log))
    ranks.finish()


def test_sharded_packed_batch_over_two_gloo_ranks():
    """The mixed batch split over two ranks: every episode is advanced by
    exactly one rank (warm-up from cycle 1, timed steps after it), the node
    updates add up to the whole batch's, and both ranks see the slowest
    rank's time."""
    from lbm_mutiwing_b200 import workloads as wl
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    eps = wl.mixed_batch(16, steps=4)
    (_, m0, n0, t0, log0), (_, m1, n1, t1, log1) = res
    assert sorted(m0 + m1) == list(range(16)) and not set(m0) & set(m1)
    assert n0 + n1 == sum(e.nx * e.ny for e in eps) * 10
    assert t0 == t1 == max(1e-9 * 10 * len(m0), 1e-9 * 10 * len(m1))
    for mine, log in ((m0, log0), (m1, log1)):
        names = [eps[i].name for i in mine]
        assert [x for x in log if x[0] != "closed"] == [(n, 1, 3) for n in names] + [(n, 4, 10) for n in names]
        assert log[-1] == ("closed", len(mine))
