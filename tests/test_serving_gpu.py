"""Device side of SAVE and of the online server.

* ``lbm_get_output`` (strided u/UU, v/UU, pressure and vorticity computed on
  the device, solution.f90:132-241) equals the same formulas applied on the
  host to the exported fields, on both paths, and the plain path's output
  agrees with the oracle's fields within the IBM tolerance;
* served FORCE replies equal the segment averages of a direct run through
  the C ABI with the same motion rows;
* a client's replies are identical alone and in a mix of concurrent clients
  (episodes are independent and deterministic), and the same whether the
  server steps episodes in packed rounds or each on its own streams.
"""
import threading

import numpy as np
import pytest

from lbm_mutiwing_b200 import api, loadgen
from lbm_mutiwing_b200 import protocol as P
from lbm_mutiwing_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def small(name, wings=2, size=(4.0, 2.0)):
    return wl.tandem_pitch_heave(name, size[0], size[1], 0.02, 100.0, -1.0, 0.0, 60, 40, n_wings=wings,
                                 x_spacing=1.5, spacing="uniform")


WORKLOADS = {"a": lambda: small("a", 2), "b": lambda: small("b", 1, (6.0, 3.0)), "c": lambda: small("c", 2, (5.0, 2.0)),
             "big": lambda: small("big", 2, (20.0, 10.0))}


def make_episode(name):
    return WORKLOADS[name]()


def host_output(ep, u, v, pre, sx, sy):
    """The output formulas (solution.f90:185-211) on host arrays (ny, nx)."""
    uu, sc = ep.uu, ep.scale
    ny, nx = u.shape
    js, is_ = np.arange(0, ny, sy), np.arange(0, nx, sx)
    vor = np.zeros((len(js), len(is_)))
    for a, j in enumerate(js):
        for b, i in enumerate(is_):
            if i == nx - 1:
                dvx = (1.5 * v[j, i] - 2.0 * v[j, i - 1] + 0.5 * v[j, i - 2]) / (uu * sc)
            elif i == 0:
                dvx = (-1.5 * v[j, i] + 2.0 * v[j, i + 1] - 0.5 * v[j, i + 2]) / (uu * sc)
            else:
                dvx = (v[j, i + 1] - v[j, i - 1]) / (uu * 2.0 * sc)
            if j == ny - 1:
                duy = (1.5 * u[j, i] - 2.0 * u[j - 1, i] + 0.5 * u[j - 2, i]) / (uu * sc)
            elif j == 0:
                duy = (-1.5 * u[j, i] + 2.0 * u[j + 1, i] - 0.5 * u[j + 2, i]) / (uu * sc)
            else:
                duy = (u[j + 1, i] - u[j - 1, i]) / (uu * 2.0 * sc)
            vor[a, b] = dvx - duy
    sel = np.ix_(js, is_)
    return u[sel] / uu, v[sel] / uu, pre[sel], vor


@pytest.mark.parametrize("prec", [api.PRECISION_FP64, api.PRECISION_FP32])
def test_output_fields_match_host_formulas(gpu_lib, prec):
    ep = small("out", 2)
    with api.Simulation(ep, prec) as s:
        s.step(6, flags=api.STEP_FIELDS)
        _, u, v, pre = s.fields()
        for sx, sy in ((2, 2), (1, 3)):
            got = s.output(sx, sy)
            want = host_output(ep, u, v, pre, sx, sy)
            for g, w in zip(got, want):
                assert np.array_equal(g, w)


def test_plain_output_matches_oracle(gpu_lib, oracle_lib):
    ep = small("out", 1)
    o = oracle_lib.Oracle(ep)
    o.run(1, 6)
    with api.Simulation(ep, api.PRECISION_FP64) as s:
        s.step(6)
        got = s.output(2, 2)
    want = host_output(ep, o.field("u"), o.field("v"), o.field("pre"), 2, 2)
    for g, w in zip(got, want):
        assert np.abs(g - w).max() <= 1e-9 * max(1.0, np.abs(w).max())


def _server(**kw):
    from lbm_mutiwing_b200.serve import Server
    srv = Server("tcp://127.0.0.1:0", make_episode, "a", precision=api.PRECISION_FP32, workers=8, **kw)
    th = threading.Thread(target=srv.serve, kwargs={"idle_timeout_s": 120}, daemon=True)
    th.start()
    return srv, th, f"tcp://127.0.0.1:{srv.port}"


def _script(name, segs=(7, 30, 12)):
    ep = make_episode(name)
    dt = ep.scale * ep.uu
    rng = np.random.default_rng(len(name))
    lines, cyc = [f"RESET 0.0 {name}"], 1
    for n in segs:
        cyc += n
        lines.append(loadgen.step_line((cyc - 1) * dt, rng.normal(0, 0.05, 3 * ep.wing_count)))
    return lines + ["STOP"]


def test_served_force_equals_direct_run(gpu_lib):
    srv, th, addr = _server()
    try:
        replies = loadgen.run_script(addr, _script("a"))
    finally:
        srv.stop()
        th.join(30)
        srv.close()
    ep = make_episode("a")
    W = ep.wing_count
    dt = ep.scale * ep.uu
    lines = _script("a")
    with api.Simulation(ep, api.PRECISION_FP32, motion_source=api.MOTION_STREAM) as s:
        ncol = 1 + 9 * W
        start = np.zeros(ncol)
        target = np.zeros(ncol)
        s.set_stream_rows(start, target)
        s.reset_sums()
        rows = s.step(1, first_cycle=1, flags=api.STEP_FIELDS)
        sm, cnt, ln = s.sums()
        want = [api.finalize_force_average(sm, cnt, ln, W, 0.0, rows[-1])]
        cyc = 2
        for line in lines[1:-1]:
            vals = [float(x) for x in line.split()[1:]]
            t = vals[0]
            start = target
            target = s.build_stream_target_row(start, t, np.array(vals))
            s.set_stream_rows(start, target)
            s.reset_sums()
            n = int(round(t / dt)) + 1 - cyc + 1
            rows = s.step(n, first_cycle=cyc, flags=api.STEP_FIELDS)
            cyc += n
            sm, cnt, ln = s.sums()
            want.append(api.finalize_force_average(sm, cnt, ln, W, t, rows[-1]))
    for r, w in zip(replies[:-1], want):
        assert r == P.force_reply(w)
    assert replies[-1] == "STATUS STOPPING"


def test_served_replies_same_alone_and_in_mix(gpu_lib):
    srv, th, addr = _server()
    try:
        alone = loadgen.run_script(addr, _script("a"), identity=b"solo")
        out = {}

        def run(k, name):
            out[k] = loadgen.run_script(addr, _script(name), identity=b"mix%d" % k)
        ths = [threading.Thread(target=run, args=(k, n)) for k, n in enumerate("abcab")]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
    finally:
        srv.stop()
        th.join(30)
        srv.close()
    assert all(r.startswith("FORCE") for r in alone[:-1])
    assert out[0] == alone and out[3] == alone
    assert out[1] == out[4]


def _mix(**kw):
    srv, th, addr = _server(**kw)
    out = {}
    try:
        def run(k, name):
            out[k] = loadgen.run_script(addr, _script(name), identity=b"mix%d" % k)
        ths = [threading.Thread(target=run, args=(k, n)) for k, n in enumerate("abcab")]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
    finally:
        srv.stop()
        th.join(30)
        srv.close()
    return out


def test_packed_rounds_equal_own_streams(gpu_lib):
    """Continuous batching in rounds of 5 steps (segments of 7, 30 and 12
    steps split across rounds, clients joining mid-segment) gives the same
    replies as every episode stepping alone on its own streams."""
    ref = _mix(packed=False)
    got = _mix(chunk=5)
    assert all(r.startswith("FORCE") for r in ref[0][:-1])
    for k in range(5):
        assert got[k] == ref[k], k


def test_admission_waits_for_free_device_memory(gpu_lib):
    """Device memory held by another user of the GPU leaves room for one
    1001 x 501 episode: a second client's RESET waits (no reply) until the
    first client's STOP frees its episode, then proceeds."""
    import torch
    import zmq
    ep = make_episode("big")
    with api.Simulation(ep, api.PRECISION_FP32, motion_source=api.MOTION_STREAM) as probe:
        actual = probe.device_bytes()
    need = api.estimate_device_bytes(ep, api.PRECISION_FP32)
    assert actual <= need
    reserve = 256 << 20
    torch.cuda.synchronize()
    free, _ = api.mem_info(0)
    slack = actual // 2      # after one episode the free memory is short of a second estimate
    hog = torch.empty(free - reserve - need - slack, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    srv, th, addr = _server(reserve_bytes=reserve)
    ctx = zmq.Context.instance()
    a, b = ctx.socket(zmq.REQ), ctx.socket(zmq.REQ)
    try:
        for sck in (a, b):
            sck.setsockopt(zmq.LINGER, 0)
            sck.connect(addr)
        a.setsockopt(zmq.RCVTIMEO, 60000)
        a.send_string("RESET 0.0 big")
        assert a.recv().decode().startswith("FORCE")
        b.setsockopt(zmq.RCVTIMEO, 1500)
        b.send_string("RESET 0.0 big")
        with pytest.raises(zmq.Again):
            b.recv()
        a.send_string("STOP")
        assert a.recv().decode() == "STATUS STOPPING"
        b.setsockopt(zmq.RCVTIMEO, 60000)
        assert b.recv().decode().startswith("FORCE")
        b.send_string("STOP")
        assert b.recv().decode() == "STATUS STOPPING"
    finally:
        a.close(0)
        b.close(0)
        srv.stop()
        th.join(30)
        srv.close()
        del hog
        torch.cuda.empty_cache()

