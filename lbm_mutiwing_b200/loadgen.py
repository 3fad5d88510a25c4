"""Simulated online clients for the episode server: scripted clients (tests)
and a seeded Poisson load of many REQ clients (serving measurements).

Each load client: RESET into a workload, then STEP segments of uniform
100..2000 lattice steps with per-wing increments of omega, x and y velocity
drawn from N(0, sigma), a SAVE with probability p_save, exponential think
times between requests (Poisson arrivals at rate_hz per client), STOP at
the end.  Latencies are measured at the client, from send to reply.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np


def run_script(endpoint: str, lines: Sequence[str], identity: Optional[bytes] = None,
               timeout_ms: int = 600000) -> List[str]:
    """Send the lines one by one over a REQ socket; the replies in order."""
    import zmq
    ctx = zmq.Context.instance()
    s = ctx.socket(zmq.REQ)
    s.setsockopt(zmq.LINGER, 0)
    s.setsockopt(zmq.RCVTIMEO, timeout_ms)
    if identity is not None:
        s.setsockopt(zmq.IDENTITY, identity)
    s.connect(endpoint)
    out = []
    try:
        for line in lines:
            s.send_string(line)
            out.append(s.recv().decode())
    finally:
        s.close(0)
    return out


def step_line(t: float, deltas: Sequence[float]) -> str:
    return "STEP " + " ".join(repr(float(x)) for x in [t, *deltas])


@dataclass
class LoadResult:
    step_latency_s: List[float] = field(default_factory=list)
    save_latency_s: List[float] = field(default_factory=list)
    node_updates: int = 0
    errors: List[str] = field(default_factory=list)
    wall_s: float = 0.0

    def percentile(self, q: float) -> float:
        return float(np.percentile(self.step_latency_s, q)) if self.step_latency_s else float("nan")

    def mlups(self) -> float:
        return self.node_updates / self.wall_s / 1e6 if self.wall_s > 0 else 0.0


def poisson_load(endpoint: str, workloads: Sequence[str], make_episode: Callable, requests_per_client: int,
                 rate_hz: float, seed: int = 20261203, seg_min: int = 100, seg_max: int = 2000,
                 sigma: float = 0.05, p_save: float = 0.05) -> LoadResult:
    """One client per workload name, all at once; returns merged results."""
    res = LoadResult()
    lock = threading.Lock()
    eps = [make_episode(w) for w in workloads]

    def client(k: int):
        import zmq
        rng = np.random.default_rng(seed + k)
        ep = eps[k]
        dt = ep.scale * ep.uu
        ctx = zmq.Context.instance()
        s = ctx.socket(zmq.REQ)
        s.setsockopt(zmq.LINGER, 0)
        s.setsockopt(zmq.RCVTIMEO, 600000)
        s.connect(endpoint)
        local = LoadResult()
        try:
            s.send_string(f"RESET 0.0 {workloads[k]}")
            r = s.recv().decode()
            if not r.startswith("FORCE"):
                local.errors.append(r)
                return
            local.node_updates += ep.nx * ep.ny
            cycle = 1
            for _ in range(requests_per_client):
                time.sleep(float(rng.exponential(1.0 / rate_hz)) if rate_hz > 0 else 0.0)
                if rng.random() < p_save:
                    t0 = time.perf_counter()
                    s.send_string("SAVE")
                    r = s.recv().decode()
                    local.save_latency_s.append(time.perf_counter() - t0)
                    continue
                n = int(rng.integers(seg_min, seg_max + 1))
                cycle += n
                deltas = rng.normal(0.0, sigma, 3 * ep.wing_count)
                t0 = time.perf_counter()
                s.send_string(step_line((cycle - 1) * dt, deltas))
                r = s.recv().decode()
                local.step_latency_s.append(time.perf_counter() - t0)
                if r.startswith("FORCE"):
                    local.node_updates += n * ep.nx * ep.ny
                else:
                    local.errors.append(r)
            s.send_string("STOP")
            s.recv()
        finally:
            s.close(0)
            with lock:
                res.step_latency_s += local.step_latency_s
                res.save_latency_s += local.save_latency_s
                res.node_updates += local.node_updates
                res.errors += local.errors

    t0 = time.perf_counter()
    th = [threading.Thread(target=client, args=(k,)) for k in range(len(workloads))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    res.wall_s = time.perf_counter() - t0
    return res
