"""Online protocol, episode session and multi-client server on the CPU, with a
stand-in simulation (the device path is covered by test_serving_gpu.py).

What is checked against the reference's driver (driver.f90, zmq_comm.f90):
command parsing and error texts, FORCE formatting (es24.16 with a length
prefix), RESET / STEP / SAVE / STOP sequencing, time alignment and
monotonicity, segment averaging of the force columns, the SAVE file, and,
for the server, concurrent clients, admission by memory and the single-client
mode's STOP.
"""
import os
import threading

import numpy as np
import pytest

from lbm_mutiwing_b200 import loadgen
from lbm_mutiwing_b200 import protocol as P
from lbm_mutiwing_b200 import session as S
from lbm_mutiwing_b200 import workloads as wl


class FakeSim:
    """Deterministic stand-in with the Simulation methods a session uses."""

    def __init__(self, ep):
        self.ep, self.W = ep, ep.wing_count
        self.nx, self.ny = ep.nx, ep.ny
        self.row_len = 4 + 12 * self.W
        self.closed = False
        self.reset()

    def reset(self):
        self.sum = np.zeros(self.row_len)
        self.cnt = 0

    def build_stream_target_row(self, start, t, delta):
        if t - start[0] < -1e-12:
            raise RuntimeError("before start")
        out = np.array(start, dtype=np.float64)
        out[0] = t
        for w in range(self.W):
            for a in range(3):
                out[1 + 9 * w + 3 * a + 1] += delta[1 + 3 * w + a]
        return out

    def set_stream_rows(self, a, b):
        self.rows = (np.array(a), np.array(b))

    def reset_sums(self):
        self.sum[:] = 0.0
        self.cnt = 0

    def step(self, n, first_cycle, rows=True, flags=0):
        dt = self.ep.scale * self.ep.uu
        out = np.zeros((n, self.row_len))
        for k in range(n):
            c = first_cycle + k
            out[k, 0] = (c - 1) * dt
            out[k, 1:] = np.sin(0.1 * c + np.arange(1, self.row_len)) + self.rows[1][1]
            self.sum = self.sum + out[k]
            self.cnt += 1
        return out

    def sums(self):
        return self.sum.copy(), self.cnt, self.row_len

    def output(self, sx, sy):
        onx, ony = (self.nx - 1) // sx + 1, (self.ny - 1) // sy + 1
        return tuple(np.full((ony, onx), float(k)) for k in range(4))

    def markers(self):
        n = int(self.ep.points_per_wing().sum())
        return np.zeros(n), np.zeros(n), None, None

    def device_bytes(self):
        return 1000 * self.nx * self.ny

    def close(self):
        self.closed = True


def small_episode(name="small", wings=2):
    return wl.tandem_pitch_heave(name, 4.0, 2.0, 0.04, 100.0, -1.0, 0.0, 40, 8, n_wings=wings,
                                 x_spacing=1.5, spacing="uniform")


def make_episode(name):
    return small_episode(name, wings=1 if name.endswith("1") else 2)


# -- protocol
def test_parse_commands_and_errors():
    assert P.parse("reset", 2) == P.Command("RESET", [0.0])
    assert P.parse("START 0.0 mix:3", 2) == P.Command("RESET", [0.0], "mix:3")
    c = P.parse("STEP 1.0d-2, 0.1 0.2 0.3 0.4 0.5 0.6 9 9", 2)
    assert c.kind == "STEP" and c.values == [0.01, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6]
    assert P.parse("save", 1).kind == "OUTPUT" and P.parse("exit", 1).kind == "STOP"
    for text, msg in [("STEP 0.1 1 2", P.ERR_STEP_VALUES), ("RESET x", P.ERR_RESET_TIME),
                      ("go", P.ERR_UNKNOWN + "GO"), ("   ", P.ERR_PARSE)]:
        with pytest.raises(P.ProtocolError) as e:
            P.parse(text, 1)
        assert str(e.value) == msg


def test_force_reply_es24_16():
    assert P.es24_16(1.0) == "1.0000000000000000E+00"
    assert P.es24_16(0.0) == "0.0000000000000000E+00"
    assert P.es24_16(-1.0e-5) == "-1.0000000000000001E-05"
    assert P.es24_16(1e100) == "1.0000000000000000+100"
    r = P.force_reply([0.5, -2.0])
    assert r == "FORCE 2 5.0000000000000000E-01 -2.0000000000000000E+00"
    assert P.parse_force_reply(r) == [0.5, -2.0]


# -- session
def test_session_sequencing_and_averages(tmp_path):
    ep = small_episode()
    sim = FakeSim(ep)
    s = S.EpisodeSession(sim, ep, str(tmp_path), 0, write_force_files=True)
    dt = ep.scale * ep.uu
    assert s.handle(P.parse("STEP 0.1 0 0 0 0 0 0", 2)) == P.error_reply(P.ERR_NEED_RESET_STEP)
    assert s.handle(P.parse("SAVE", 2)) == P.error_reply(P.ERR_NEED_RESET_SAVE)
    assert s.handle(P.parse("RESET 0.5", 2)) == P.error_reply(P.ERR_RESET_NONZERO)
    r = s.handle(P.parse("RESET", 2))
    vals = P.parse_force_reply(r)
    assert len(vals) == 4 + 12 * 2 and vals[0] == 0.0 and s.n == 2
    # a 7-step segment: averaged force columns, last-step motion columns, end time
    t = 7 * dt
    r = s.handle(P.parse(f"STEP {t!r} 0.1 0 0 0 0 0", 2))
    vals = np.array(P.parse_force_reply(r))
    rows = s.last_rows
    assert rows.shape[0] == 7 and s.n == 9
    W = 2
    np.testing.assert_array_equal(vals[1:1 + 3 * W + 3], np.cumsum(rows, axis=0)[-1][1:1 + 3 * W + 3] / 7)
    np.testing.assert_array_equal(vals[1 + 3 * W + 3:], rows[-1][1 + 3 * W + 3:])
    assert vals[0] == t
    # misaligned, backwards, before the segment start
    assert s.handle(P.parse(f"STEP {t + dt / 3!r} 0 0 0 0 0 0", 2)) == P.error_reply(P.ERR_ALIGN)
    assert s.handle(P.parse(f"STEP {t - dt!r} 0 0 0 0 0 0", 2)) == P.error_reply(P.ERR_STEP_BEFORE_START)
    assert s.handle(P.parse(f"STEP {t!r} 0 0 0 0 0 0", 2)) == P.error_reply(P.ERR_BACKWARDS)
    # a failed STEP leaves the segment rows as they were
    assert s.target_row[0] == t
    r = s.handle(P.parse("SAVE", 2))
    assert r == P.status_reply("FLOW_SAVED F8.dat")
    path = tmp_path / "episode_1" / "F8.dat"
    lines = path.read_text().splitlines()
    onx, ony = (ep.nx - 1) // 2 + 1, (ep.ny - 1) // 2 + 1
    npts = int(ep.points_per_wing().sum())
    assert len(lines) == 2 + onx * ony + 1 + npts + 2 + (npts - 2)
    assert len(lines[2]) == 8 * 16
    force_lines = (tmp_path / "force_episode_1.dat").read_text().splitlines()
    assert len(force_lines) == 1 + 7 and len(force_lines[0]) == 15 * (4 + 12 * W)
    assert s.handle(P.parse("STOP", 2)) == P.status_reply("STOPPING")


# -- server
def _server(**kw):
    from lbm_mutiwing_b200.serve import Server
    kw.setdefault("free_memory", None)
    factory = kw.pop("sim_factory", lambda ep, p, d: FakeSim(ep))
    srv = Server("tcp://127.0.0.1:0", make_episode, "small2", sim_factory=factory, **kw)
    th = threading.Thread(target=srv.serve, kwargs={"idle_timeout_s": 30}, daemon=True)
    th.start()
    return srv, th, f"tcp://127.0.0.1:{srv.port}"


def _script(dt, n_seg=4, wings=2):
    lines, cyc = ["RESET"], 1
    for k in range(n_seg):
        cyc += 5 + k
        lines.append(loadgen.step_line((cyc - 1) * dt, [0.01 * k] * (3 * wings)))
    return lines + ["STOP"]


def test_server_clients_alone_and_together():
    ep = make_episode("small2")
    dt = ep.scale * ep.uu
    srv, th, addr = _server()
    try:
        alone = loadgen.run_script(addr, _script(dt), identity=b"a")
        out = {}
        ths = [threading.Thread(target=lambda k=k: out.__setitem__(k, loadgen.run_script(addr, _script(dt),
                                                                                          identity=b"c%d" % k)))
               for k in range(4)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        for k in range(4):
            assert out[k] == alone
        assert alone[-1] == "STATUS STOPPING" and all(r.startswith("FORCE") for r in alone[:-1])
    finally:
        srv.stop()
        th.join(10)
        srv.close()


class FakeDevice:
    """Device memory of FakeSim episodes: free = total - live episodes."""

    def __init__(self, total):
        self.total, self.live = total, []

    def factory(self, ep, precision, device):
        sim = FakeSim(ep)
        self.live.append(sim)
        return sim

    def free(self):
        return self.total - sum(s.device_bytes() for s in self.live if not s.closed)


def _two_clients_one_fits(**kw):
    """Client a's RESET is admitted, b's waits until a's STOP frees memory."""
    srv, th, addr = _server(**kw)
    try:
        import zmq
        ctx = zmq.Context.instance()
        a, b = ctx.socket(zmq.REQ), ctx.socket(zmq.REQ)
        for s in (a, b):
            s.setsockopt(zmq.LINGER, 0)
            s.setsockopt(zmq.RCVTIMEO, 20000)
            s.connect(addr)
        a.send_string("RESET")
        assert a.recv().decode().startswith("FORCE")
        b.send_string("RESET")
        with pytest.raises(zmq.Again):
            b.setsockopt(zmq.RCVTIMEO, 500)
            b.recv()
        a.send_string("STOP")
        assert a.recv().decode() == "STATUS STOPPING"
        b.setsockopt(zmq.RCVTIMEO, 20000)
        assert b.recv().decode().startswith("FORCE")
        a.close(0)
        b.close(0)
    finally:
        srv.stop()
        th.join(10)
        srv.close()


def test_server_admission_waits_for_free_device_memory():
    ep = make_episode("small2")
    per = 1000 * ep.nx * ep.ny                      # a FakeSim episode's device bytes
    dev = FakeDevice(total=(3 * per) // 2 + (1 << 20))   # room for one episode and the reserve
    _two_clients_one_fits(sim_factory=dev.factory, free_memory=dev.free, reserve_bytes=1 << 20,
                          estimate=lambda e, p: 1000 * e.nx * e.ny)


def test_server_admission_within_a_byte_budget():
    ep = make_episode("small2")
    per = 1000 * ep.nx * ep.ny
    _two_clients_one_fits(budget_bytes=per + 1, estimate=lambda e, p: 1000 * e.nx * e.ny)


def test_single_client_mode_stops_on_stop():
    from lbm_mutiwing_b200.serve import Server
    srv = Server("tcp://127.0.0.1:0", make_episode, "small2", single=True,
                 sim_factory=lambda ep, p, d: FakeSim(ep), free_memory=None)
    th = threading.Thread(target=srv.serve, daemon=True)
    th.start()
    addr = f"tcp://127.0.0.1:{srv.port}"
    r = loadgen.run_script(addr, ["STEP 1 0 0 0 0 0 0", "RESET", "STOP"])
    th.join(10)
    assert not th.is_alive()
    srv.close()
    assert r[0] == P.error_reply(P.ERR_NEED_RESET_STEP)
    assert r[1].startswith("FORCE 28 ") and r[2] == "STATUS STOPPING"
