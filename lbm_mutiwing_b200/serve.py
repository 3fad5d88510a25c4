"""Online serving front end: the reference's ZeroMQ driver (driver.f90:59-408,
zmq_comm.f90) turned into a request loop for many clients with continuous
batching.

* One ROUTER socket; every client (ZeroMQ identity) owns one episode, kept
  resident in HBM between its requests.
* Requests are executed by a pool of worker threads.  The lattice steps of
  FP32 episodes go to one continuous batcher (``batch.PackedStepper``): every
  step is one packed launch per kernel over all clients' episodes in flight,
  in rounds of at most ``chunk`` steps, and a request that arrives meanwhile
  joins at the next round -- it does not wait for the others' segments to
  end.  FP64 episodes (and ``packed=False``) step on their own CUDA streams.
* Admission by free device memory: a RESET that creates an episode is
  admitted when the episode's estimated device memory fits in the device's
  free memory (cudaMemGetInfo) less a reserve and less what episodes admitted
  but not yet created will take; otherwise it waits until running episodes
  end (STOP) and free their memory.  Once created, an episode counts with
  the memory its handle actually holds.  An optional byte budget bounds the
  resident episodes as well.
* Replies are the reference's text replies (``protocol``); per-request
  latency is recorded for p50 / p99.
* ``single=True`` is the reference's one-client driver on a REP socket: one
  episode, STOP ends the server.

Episodes are independent and deterministic, so a client's replies are the
same alone and in any mix.
"""
from __future__ import annotations

import os
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional, Tuple

import numpy as np

from . import protocol as P
from .session import EpisodeSession


@dataclass
class RequestStat:
    kind: str
    latency_s: float
    node_updates: int


@dataclass
class _Client:
    ident: bytes
    session: Optional[EpisodeSession] = None
    workload: Optional[str] = None
    nodes: int = 0
    queue: Deque[Tuple[float, str]] = field(default_factory=deque)
    busy: bool = False
    bytes: int = 0
    reserved: int = 0        # admission reservation until the episode exists


def _default_sim_factory(ep, precision, device):
    from .api import MOTION_STREAM, Simulation
    return Simulation(ep, precision, motion_source=MOTION_STREAM, device=device)


class Server:
    """Multi-client episode server.

    make_episode(name) -> Episode builds the episode a RESET names (the
    default workload when the RESET names none).  Admission: free_memory()
    (default: the device's free bytes, lbm_mem_info; None disables the
    check) less reserve_bytes must hold the new episode's estimate
    (estimate(ep, precision), default api.estimate_device_bytes) plus the
    estimates of episodes admitted and not yet created; budget_bytes (None:
    no bound) also bounds the memory the resident episodes hold."""

    def __init__(self, endpoint: str, make_episode: Callable, default_workload: str, precision: int = 1,
                 device: int = 0, workers: int = 64, out_dir: Optional[str] = None,
                 budget_bytes: Optional[int] = None, single: bool = False, write_force_files: bool = False,
                 sim_factory: Optional[Callable] = None, packed: bool = True, chunk: int = 200,
                 free_memory: Optional[Callable[[], int]] = "device", reserve_bytes: int = 1 << 30,
                 estimate: Optional[Callable] = None):
        import zmq
        self.zmq = zmq
        self.endpoint = endpoint
        self.make_episode = make_episode
        self.default_workload = default_workload
        self.precision = precision
        self.device = device
        self.out_dir = out_dir
        self.budget = budget_bytes
        if free_memory == "device":
            from .api import mem_info
            free_memory = lambda: mem_info(device)[0]   # noqa: E731
        self.free_memory = free_memory
        self.reserve = reserve_bytes
        if estimate is None:
            from .api import estimate_device_bytes as estimate
        self.estimate = estimate
        self.pending_bytes = 0          # admitted RESETs whose episode is not created yet
        self.single = single
        self.write_force_files = write_force_files
        self.sim_factory = sim_factory or _default_sim_factory
        # packed stepping needs the library's simulations on the FP32 path
        self.packed = packed and sim_factory is None and precision != 0 and not single
        self.chunk = chunk
        self._stepper = None
        self.ctx = zmq.Context.instance()
        self.sock = self.ctx.socket(zmq.REP if single else zmq.ROUTER)
        self.sock.setsockopt(zmq.LINGER, 0)
        self.sock.bind(endpoint)
        self.port = None
        ep = self.sock.getsockopt(zmq.LAST_ENDPOINT).decode()
        if ep.startswith("tcp://"):
            self.port = int(ep.rsplit(":", 1)[1])
        self.pool = ThreadPoolExecutor(max_workers=1 if single else workers)
        self.done: Deque[Tuple[bytes, str, RequestStat]] = deque()
        self.wake_addr = f"inproc://lbm-wake-{id(self)}"
        self.wake_pull = self.ctx.socket(zmq.PULL)
        self.wake_pull.bind(self.wake_addr)
        self.clients: Dict[bytes, _Client] = {}
        self.waiting_admission: Deque[bytes] = deque()
        self.resident_bytes = 0
        self.stats: List[RequestStat] = []
        self.episode_counter = 0
        self.stopped = threading.Event()
        self.lock = threading.Lock()
        self._tls = threading.local()

    # -- worker side
    def _wake(self):
        s = getattr(self._tls, "push", None)
        if s is None:
            s = self.ctx.socket(self.zmq.PUSH)
            s.setsockopt(self.zmq.LINGER, 0)
            s.connect(self.wake_addr)
            self._tls.push = s
        s.send(b"")

    def _run(self, c: _Client, t_recv: float, text: str):
        wc = c.session.W if c.session is not None else None
        node_updates = 0
        kind = "?"
        try:
            # without an episode only RESET and STOP are meaningful
            cmd = P.parse(text, wc if wc is not None else 0)
            kind = cmd.kind
            if cmd.kind == P.CMD_RESET:
                reply = self._reset(c, cmd)
            elif c.session is None:
                reply = P.error_reply(P.ERR_NEED_RESET_SAVE if cmd.kind == P.CMD_OUTPUT
                                      else P.ERR_NEED_RESET_STEP) if cmd.kind != P.CMD_STOP \
                    else P.status_reply(P.STATUS_STOPPING)
                if cmd.kind == P.CMD_STOP:
                    self._release(c)
            else:
                before = c.session.steps_run
                reply = c.session.handle(cmd)
                node_updates = (c.session.steps_run - before) * c.nodes
                if cmd.kind == P.CMD_STOP:
                    self._release(c)
        except P.ProtocolError as e:
            reply = P.error_reply(str(e))
        except Exception as e:  # library errors become ERROR replies (driver.f90:135-138)
            reply = P.error_reply(str(e))
        if c.reserved:   # an admitted RESET that created no episode gives its reservation back
            with self.lock:
                self.pending_bytes -= c.reserved
            c.reserved = 0
        st = RequestStat(kind, time.perf_counter() - t_recv, node_updates)
        self.done.append((c.ident, reply, st))
        self._wake()

    def _reset(self, c: _Client, cmd: P.Command) -> str:
        name = cmd.workload or c.workload or self.default_workload
        if c.session is None or name != c.workload:
            self._release(c)
            ep = self.make_episode(name)
            try:
                sim = self.sim_factory(ep, self.precision, self.device)
            finally:
                with self.lock:   # the admission reservation ends with the creation
                    self.pending_bytes -= c.reserved
                c.reserved = 0
            with self.lock:
                self.episode_counter += 1
                idx = self.episode_counter - 1
            out = self.out_dir
            if out is not None and not self.single:
                out = os.path.join(out, f"client_{idx}")
            c.session = EpisodeSession(sim, ep, out, 0, self.write_force_files, stepper=self._get_stepper())
            c.workload = name
            c.nodes = ep.nx * ep.ny
            nb = int(sim.device_bytes()) if hasattr(sim, "device_bytes") else 0
            with self.lock:
                self.resident_bytes += nb - c.bytes
            c.bytes = nb
        return c.session.handle(cmd)

    def _get_stepper(self):
        if not self.packed:
            return None
        with self.lock:
            if self._stepper is None:
                from .batch import PackedStepper
                self._stepper = PackedStepper(self.device, self.chunk)
            return self._stepper.step

    def _release(self, c: _Client):
        if c.session is not None:
            c.session.close()
            sim = c.session.sim
            if hasattr(sim, "close"):
                sim.close()
            c.session = None
        with self.lock:
            self.resident_bytes -= c.bytes
        c.bytes = 0
        c.workload = None

    # -- admission
    def _need(self, c: _Client, text: str) -> int:
        """Estimated bytes of the episode a RESET would create (0 when it
        keeps the client's episode)."""
        toks = text.split()
        name = toks[2] if len(toks) > 2 else (c.workload or self.default_workload)
        if c.session is not None and name == c.workload:
            return 0
        try:
            ep = self.make_episode(name)
        except Exception:
            return 0          # the RESET fails on its own and takes no memory
        return int(self.estimate(ep, self.precision))

    def _admit(self, c: _Client, text: str) -> bool:
        """Reserve the RESET's memory if it fits; False if it must wait."""
        need = self._need(c, text)
        if need == 0:
            return True
        with self.lock:
            if self.budget is not None and self.resident_bytes - c.bytes + need > self.budget:
                return False
            if self.free_memory is not None:
                # a client's own episode is freed before its new one is made
                if self.pending_bytes + need > self.free_memory() + c.bytes - self.reserve:
                    return False
            self.pending_bytes += need
            c.reserved = need
        return True

    # -- main loop
    def _dispatch(self, c: _Client):
        if c.busy or not c.queue:
            return
        t_recv, text = c.queue[0]
        first = text.strip().split()[:1]
        if first and first[0].upper() in ("RESET", "START") and not self._admit(c, text):
            if c.ident not in self.waiting_admission:
                self.waiting_admission.append(c.ident)
            return
        c.queue.popleft()
        c.busy = True
        self.pool.submit(self._run, c, t_recv, text)

    def _send(self, ident: bytes, reply: str):
        if self.single:
            self.sock.send_string(reply)
        else:
            self.sock.send_multipart([ident, b"", reply.encode()])

    def serve(self, max_requests: Optional[int] = None, idle_timeout_s: Optional[float] = None):
        """Run until a STOP (single mode), stop(), max_requests replies, or
        idle_timeout_s without any request."""
        zmq = self.zmq
        poller = zmq.Poller()
        poller.register(self.sock, zmq.POLLIN)
        poller.register(self.wake_pull, zmq.POLLIN)
        replies = 0
        last = time.perf_counter()
        while not self.stopped.is_set():
            ev = dict(poller.poll(50))
            now = time.perf_counter()
            if self.sock in ev:
                if self.single:
                    ident, text = b"single", self.sock.recv().decode(errors="replace")
                else:
                    parts = self.sock.recv_multipart()
                    ident, text = parts[0], parts[-1].decode(errors="replace")
                c = self.clients.get(ident)
                if c is None:
                    c = self.clients[ident] = _Client(ident)
                c.queue.append((now, text))
                self._dispatch(c)
                last = now
            if self.wake_pull in ev:
                while True:
                    try:
                        self.wake_pull.recv(zmq.NOBLOCK)
                    except zmq.Again:
                        break
            while self.done:
                ident, reply, st = self.done.popleft()
                self._send(ident, reply)
                self.stats.append(st)
                replies += 1
                c = self.clients[ident]
                c.busy = False
                if self.single and reply == P.status_reply(P.STATUS_STOPPING):
                    self.stopped.set()
                # freed memory may admit waiting episodes
                for _ in range(len(self.waiting_admission)):
                    w = self.waiting_admission.popleft()
                    self._dispatch(self.clients[w])
                self._dispatch(c)
                last = time.perf_counter()
            if max_requests is not None and replies >= max_requests:
                break
            if idle_timeout_s is not None and time.perf_counter() - last > idle_timeout_s and \
                    not any(cl.busy for cl in self.clients.values()):
                break

    def stop(self):
        self.stopped.set()

    def close(self):
        self.pool.shutdown(wait=True)
        for c in list(self.clients.values()):
            self._release(c)
        if self._stepper is not None:
            self._stepper.close()
            self._stepper = None
        self.sock.close(0)
        self.wake_pull.close(0)

    # -- metrics
    def step_latency_percentiles(self) -> Tuple[float, float]:
        lat = sorted(s.latency_s for s in self.stats if s.kind == P.CMD_STEP)
        if not lat:
            return float("nan"), float("nan")
        return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


def main(argv=None):
    """Reference-compatible entry: LBM_ZMQ_ENDPOINT (default tcp://*:5555),
    one REP client and one episode unless --multi is given."""
    import argparse
    from . import workloads as wl
    p = argparse.ArgumentParser(description="LBM_Mutiwing online server")
    p.add_argument("--endpoint", default=os.environ.get("LBM_ZMQ_ENDPOINT", "tcp://*:5555"))
    p.add_argument("--workload", default="4000x2000")
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--multi", action="store_true", help="many clients on a ROUTER socket")
    p.add_argument("--workers", type=int, default=64)
    p.add_argument("--out-dir", default="output")
    p.add_argument("--force-files", action="store_true")
    a = p.parse_args(argv)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    srv = Server(a.endpoint, wl.by_name, a.workload, 1 if a.precision == "fp32" else 0,
                 workers=a.workers, out_dir=a.out_dir, single=not a.multi, write_force_files=a.force_files)
    try:
        srv.serve()
    finally:
        srv.close()


if __name__ == "__main__":
    main()
