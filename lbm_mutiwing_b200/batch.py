"""Many resident episodes advanced side by side on one GPU.

Every episode keeps its lattice, markers and geometry in HBM.  Two ways to
advance them together:

* packed (``advance_packed``, ``PackedStepper``): one ``lbm_batch_step``
  call steps every episode, each kernel of a step being one launch over all
  episodes still stepping -- the form the server uses for FP32 episodes;
* streams (``advance_together``): a pool of host threads submits each
  episode's own step segments (CUDA graphs on its own streams).

``PackedStepper`` is the server's continuous batcher: worker threads hand
it (episode, steps) requests, a GPU thread advances all pending requests in
rounds of at most ``chunk`` steps, and requests that arrive meanwhile join
at the next round.  Stepping a segment in rounds gives the same bits as in
one call (the cycle counter, force sums and geometry continue across
calls; fields and diagnostics are requested on the last round only).
"""
from __future__ import annotations

import os
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence, Tuple

import numpy as np

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


def advance_packed(sims: Sequence[api.Simulation], steps: int, first_cycle: int = 1,
                   packed: Optional[api.Batch] = None) -> float:
    """Advance every episode by steps in packed launches; wall seconds."""
    own = packed is None
    b = api.Batch(sims[0].cfg.device) if own else packed
    try:
        t0 = time.perf_counter()
        b.step(sims, steps, first_cycles=[first_cycle] * len(sims), rows=False)
        return time.perf_counter() - t0
    finally:
        if own:
            b.close()


class _StepRequest:
    def __init__(self, sim, n, first, flags, rows):
        self.sim, self.left, self.next, self.flags, self.want_rows = sim, n, first, flags, rows
        self.parts: List[np.ndarray] = []
        self.error: Optional[BaseException] = None
        self.done = threading.Event()


class PackedStepper:
    """Continuous batching of step requests over FP32 episodes (see the
    module text).  ``step`` has the signature of ``Simulation.step``.
    ``batch`` (default: an ``api.Batch`` on ``device``) is anything with
    ``step(sims, n_steps, first_cycles=, rows=, flags=)`` and ``close()``."""

    def __init__(self, device: int = 0, chunk: int = 200, batch=None):
        self.chunk = chunk
        self.batch = batch if batch is not None else api.Batch(device)
        self.cv = threading.Condition()
        self.pending: List[_StepRequest] = []
        self.closed = False
        self.rounds = 0
        self.thread = threading.Thread(target=self._loop, name="lbm-packed-stepper", daemon=True)
        self.thread.start()

    def step(self, sim, n_steps: int = 1, first_cycle: Optional[int] = None, rows: bool = True,
             flags: int = 0) -> Optional[np.ndarray]:
        first = sim.cycle if first_cycle is None else first_cycle
        if n_steps <= 0:
            return sim.step(n_steps, first_cycle=first, rows=rows, flags=flags)
        r = _StepRequest(sim, int(n_steps), int(first), int(flags), rows)
        with self.cv:
            if self.closed:
                raise api.LbmError("stepper closed")
            self.pending.append(r)
            self.cv.notify()
        r.done.wait()
        if r.error is not None:
            raise r.error
        sim.cycle = first + n_steps
        return np.concatenate(r.parts) if rows else None

    def _loop(self):
        active: List[_StepRequest] = []
        while True:
            with self.cv:
                while not self.pending and not active and not self.closed:
                    self.cv.wait()
                if self.closed and not self.pending and not active:
                    return
                active.extend(self.pending)
                self.pending.clear()
            ks = [min(r.left, self.chunk) for r in active]
            fl = [r.flags if k == r.left else 0 for r, k in zip(active, ks)]
            try:
                if len(active) == 1:   # one episode: its own step graphs
                    r = active[0]
                    outs = [r.sim.step(ks[0], first_cycle=r.next, rows=True, flags=fl[0])]
                else:
                    outs = self.batch.step([r.sim for r in active], ks, first_cycles=[r.next for r in active],
                                           rows=True, flags=fl)
                failed = [None] * len(active)
            except api.BatchStepError as e:
                # episodes that failed their status check fail alone; the
                # others were stepped and keep their rows
                failed = [api.LbmError(m) if c else None for c, m in zip(e.rcs, e.messages)]
                outs = list(e.outs)
                if not any(failed):
                    failed = [api.LbmError(str(e))] * len(active)
            except Exception as e:   # noqa: BLE001 - handed to the waiting requests
                failed = [e] * len(active)
                outs = [None] * len(active)
            self.rounds += 1
            still = []
            for r, k, o, err in zip(active, ks, outs, failed):
                if err is not None:
                    r.error = err
                    r.done.set()
                    continue
                if o is not None:
                    r.parts.append(o)
                r.left -= k
                r.next += k
                if r.left == 0:
                    r.done.set()
                else:
                    still.append(r)
            active = still

    def close(self):
        with self.cv:
            self.closed = True
            self.cv.notify()
        self.thread.join(60)
        self.batch.close()


class PackedEngine:
    """The packed engine of one GPU for ``sharded_packed_run``: creates FP32
    episodes on ``device`` and advances them with ``lbm_batch_step``."""

    def __init__(self, device: int = 0):
        self.device = device
        self.batch = None

    def create(self, eps: Sequence) -> List[api.Simulation]:
        self.batch = api.Batch(self.device)
        return create(eps, api.PRECISION_FP32, device=self.device)

    def advance(self, sims, steps: int, first_cycle: int) -> float:
        return advance_packed(sims, steps, first_cycle=first_cycle, packed=self.batch)

    def close(self, sims) -> None:
        for s in sims:
            s.close()
        if self.batch is not None:
            self.batch.close()
            self.batch = None


def sharded_packed_run(eps: Sequence, steps: int, warmup: int, rank: int, world: int, engine=None,
                       barrier=None) -> Tuple[List[int], int, float]:
    """This rank's shard of the episodes (balanced by node count with
    ``ranks.shard``; the shards partition the episodes and need no data
    exchange) advanced ``warmup`` untimed and then ``steps`` timed packed
    steps on this rank's GPU.  Returns (episode indices, node updates of the
    timed steps, wall seconds of the timed call, which returns once the
    device work is done).  ``barrier`` (optional) runs just before the timed
    call on every rank."""
    from . import ranks
    mine = ranks.shard([float(e.nx * e.ny) for e in eps], world)[rank]
    engine = engine if engine is not None else PackedEngine()
    sims = engine.create([eps[i] for i in mine])
    try:
        if sims:
            engine.advance(sims, warmup, 1)
        if barrier is not None:
            barrier()
        seconds = engine.advance(sims, steps, 1 + warmup) if sims else 0.0
    finally:
        engine.close(sims)
    return mine, sum(eps[i].nx * eps[i].ny for i in mine) * steps, seconds


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
