"""Benchmark: MLUPS of the LBM_Mutiwing time step on B200.

Default workload: the 4000x2000 two-wing case (4001 x 2001 nodes, dx = 0.01,
Re 1000, two NACA0012 wings with 200 markers each at equal arc length,
analytic pitch/heave motion), FP32 deviation storage, FP64 immersed boundary
and force reductions.  A "step" is one lattice time step (evolution,
solution.f90:272) of one episode; with N GPUs every rank advances its own
episode (episodes are independent: weak scaling, no collective on the data
path; the only collectives are the timing barrier and max).

value  = whole-job MLUPS = sum over ranks of nx*ny*K / max-over-ranks time of
         K steps, timed with CUDA events on the library's stream, state
         resident in HBM.  The K-step timed call is repeated back to back
         for at least 1.2 s (and at least 3 times) while nvidia-smi samples
         the clocks; every repetition is exactly K steps between a barrier
         and a device synchronisation, and the median repetition is reported.
e2e    = the same metric through the online STEP path of the C ABI: per
         segment of 50 steps, the segment's two motion rows go host -> device
         and every step's force row comes back device -> host, both inside the
         timed region.
roofline: the dominant kernel's algorithmic traffic over its mean CUDA-event
         time, against the measured HBM copy bandwidth.  FP32 path: the
         two-step pass's far-tile kernel, 9 reads of step n + 9 writes of
         step n + 2, 4 bytes each, per node of the far tiles it processed
         (64 x 8 nodes a tile, 64 x 12 from 32 Mi lattice nodes on);
         whole_step_frac counts 36 bytes per node and step (a pass moves
         each node's distributions once for two steps),
         one_step_equivalent_frac 72 (the bytes a one-step scheme moves at
         the same step rate).
The distribution planes (2 x 288 MB) exceed the 126 MB L2, so no separate L2
flush is needed between steps.

Extra keys: plain_fp64 (the plain FP64 path on the same workload),
parity (both GPU paths against the CPU FP64 oracle over the first steps of
the workload: relative L2 of u, v, p, vorticity and the segment-averaged
force error), serving (64 mixed episodes packed, on their own streams and
one at a time; served STEP latency), batched_sharded (N > 1: the mixed
batch split over the ranks).

--impl reference times the CPU oracle (the C++ FP64 restatement of the
reference's Fortran, which cannot be compiled here) on the same workload with
all host threads, rank 0 only: W untimed and exactly K timed steps.

--gpus N without a torchrun environment relaunches this script under
torch.distributed.run with N processes (one per GPU).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# many episodes' streams in flight (the batched and served measurements)
# need more hardware work queues than the default 8; read at context creation
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, ROOT)

METRIC = "MLUPS (lattice node updates per second / 1e6)"
UNIT = "MLUPS"
SEG = 50
CLOCK_WINDOW_S = 1.2       # timed repetitions span at least this long
MAX_TIMED_STEPS = 12000    # bound on the repeated timed steps
MARKERS = ("NACA0012 markers at equal arc length along each surface (1.0-1.02 lattice spacings at "
           "200 markers on a 100-node chord), not the configuration's cosine spacing: cosine spacing puts "
           "trailing-edge markers 0.025 spacings apart, where the immersed-boundary system is singular and "
           "the reference's algorithm (the FP64 oracle) diverges after 1157 steps of the 800x400 case")


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--workload", default="4000x2000", choices=["800x400", "4000x2000", "16000x8000"])
    p.add_argument("--pass-tiles", default="auto", choices=["auto", "short", "tall"],
                   help="tile shape of the two-step passes: by lattice size (64 x 12 from 32 Mi nodes, else "
                        "64 x 8), or forced either way")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-serving", action="store_true", help="skip the batched and served measurements")
    p.add_argument("--packed", action="store_true",
                   help="only the 64-episode mixed batch in packed launches (lbm_batch_step), split over the "
                        "ranks: W warm-up steps, then K timed steps; one JSON line")
    return p.parse_args(argv)


def workload(name, steps):
    from lbm_mutiwing_b200 import workloads as wl
    if name == "800x400":
        return wl.tandem_800x400(steps=steps)
    if name == "16000x8000":
        return wl.formation_16000x8000(steps=steps)
    return wl.tandem_4000x2000(steps=steps)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch(argv, gpus):
    """One process per GPU under torch.distributed.run (bounded by timeout)."""
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={gpus}", "--master-addr", "127.0.0.1", f"--master-port={free_port()}",
           os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


class Clocks:
    """nvidia-smi samples (every 100 ms, time-stamped) kept only between
    begin() and end()."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.fh = None
        self.path = tempfile.mktemp(suffix=".csv")
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # wait for the sampler's first row (nvidia-smi takes a moment to start)
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def begin(self):
        self.t0 = datetime.datetime.now()

    def end(self):
        self.t1 = datetime.datetime.now()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.fh:
            self.fh.close()

    def summary(self):
        try:
            rows = []
            for line in open(self.path).read().strip().splitlines():
                r = [x.strip() for x in line.split(",")]
                if len(r) < 10:
                    continue
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f")
                if self.t0 and self.t1 and self.t0 <= ts <= self.t1:
                    rows.append(r)
            sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
            mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for k, nm in enumerate(names):
                    if r[6 + k].lower() == "active":
                        reasons.add(nm)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                    "reasons": sorted(reasons), "samples": len(rows)}
        except Exception as e:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "error": str(e)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload_name, kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        d = json.load(open(p))
        return d.get(kernel, {}).get(workload_name)
    except Exception:
        return None


# Kernels of one step with wings:
#   fused FP32 single step: geometry, claim, count, scan, list, assemble,
#               factor (a later step's geometry) | rhs, solve, spread, close |
#               bulk | far field
#   fused FP32 two-step pass: the geometry of two later steps (2 x 7) | two
#               chains (2 x 4) | two far fields | ring | near tiles | far tiles
#   plain FP64: geometry, claim, count, scan, list, assemble, factor, stream,
#               moments, ustar, rhs, solve, spread, finish, forces, collide,
#               far field, advance
KERNELS_PER_STEP = {"fp32": 13, "fp64": 18}
KERNELS_PER_PASS = 27


def kernels_in_call(k, precision):
    """Kernels one lbm_step call of k steps (no field request) launches: on
    the FP32 path every step runs in a pass but one of an odd count."""
    if precision != "fp32":
        return k * KERNELS_PER_STEP["fp64"]
    passes = k // 2
    return passes * KERNELS_PER_PASS + (k - 2 * passes) * KERNELS_PER_STEP["fp32"]


def config_of(ep, storage, world):
    return {"workload": ep.name, "nodes": ep.nx * ep.ny, "wings": ep.wing_count,
            "markers_per_wing": int(ep.markers[0].shape[0] - 1), "markers": MARKERS, "storage": storage,
            "l2": "distribution planes exceed the 126 MB L2; no flush",
            "parallelism": f"{world} independent episodes (one per GPU)"}


def oracle_steps(ep, threads, steps, warmup=1):
    """The oracle on the full workload: warmup untimed steps, then exactly
    `steps` timed steps; returns (MLUPS, seconds, oracle) with the oracle
    still open (its state after warmup + steps)."""
    from oracle import oracle
    oracle.build()
    o = oracle.Oracle(ep, nthreads=threads)
    rows = [o.step(c) for c in range(1, warmup + 1)]
    t0 = time.perf_counter()
    rows += [o.step(c) for c in range(warmup + 1, warmup + steps + 1)]
    dt = time.perf_counter() - t0
    return ep.nx * ep.ny * steps / dt / 1e6, dt, o, np.stack(rows)


def run_reference(args):
    """The reference's algorithm on the host cores: the oracle (a C++ FP64
    restatement of the Fortran, which has no compiler here), all threads, on
    the same workload: W untimed, then K timed steps (fewer only when K
    steps would take more than about four minutes; the line says so)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    K, Wm = max(1, args.steps), max(3, args.warmup)
    ep = workload(args.workload, K + Wm + 4)
    # a one-step probe bounds the timed sample
    from oracle import oracle
    oracle.build()
    probe = oracle.Oracle(ep, nthreads=threads)
    probe.step(1)
    t0 = time.perf_counter()
    probe.step(2)
    per = time.perf_counter() - t0
    probe.close()
    steps = K if per * (K + Wm) <= 240.0 else max(2, int(240.0 / per) - Wm)
    mlups, dt, o, _ = oracle_steps(ep, threads, steps, warmup=Wm)
    o.close()
    line = {"metric": METRIC, "value": mlups, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": Wm, "ms_per_step": dt / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded NACA0012 geometry, analytic pitch/heave motion)",
            "config": config_of(ep, "fp64 plain (host)", 1),
            "cpu_baseline": {"value": mlups, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} full steps of {ep.name} after {Wm} untimed steps ({dt:.1f} s)"},
            "e2e": {"value": mlups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if steps != K:
        line["steps_note"] = f"{K} steps would take about {per * K:.0f} s; timed {steps}"
    print(json.dumps(line))


def parity_and_cpu_baseline(ep_name, budget_s=15.0):
    """The oracle on all host cores over the first steps of the workload
    (about budget_s seconds; its timed steps are the CPU baseline), and both
    GPU paths over the same steps: relative L2 of u, v, p and vorticity
    after the last step and the error of the segment-averaged per-wing
    forces over the steps, each path against the oracle."""
    from lbm_mutiwing_b200 import api
    from oracle import fields as F
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.build()
    ep = workload(ep_name, 400)
    probe = oracle.Oracle(ep, nthreads=threads)
    probe.step(1)
    t0 = time.perf_counter()
    probe.step(2)
    per = time.perf_counter() - t0
    probe.close()
    n = int(min(200, max(4, budget_s / max(per, 1e-6))))
    mlups, dt, o, rows_o = oracle_steps(ep, threads, n - 1, warmup=1)
    u_o, v_o, p_o = o.field("u"), o.field("v"), o.field("pre")
    o.close()
    out = {"steps": n, "oracle_threads": threads,
           "force": "segment-averaged per-wing Fx, Fy, M over the steps, max relative error per quantity",
           "fields": "relative L2 over all nodes after the last step"}
    W = ep.wing_count
    for prec, key in ((api.PRECISION_FP32, "fp32"), (api.PRECISION_FP64, "fp64")):
        with api.Simulation(ep, prec) as s:
            rows = s.step(n, flags=api.STEP_FIELDS)
            _, u, v, p = s.fields()
        e = F.field_errors(u, v, p, u_o, v_o, p_o, ep.uu, ep.scale)
        e["force_max_rel"] = F.force_error(F.segment_average(rows, W), F.segment_average(rows_o, W))
        out[key] = e
    cpu = {"value": mlups, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"{n - 1} full steps of {ep.name} after 1 untimed step ({dt:.1f} s)"}
    return out, cpu


def serving_metrics(steps=200, requests=3, rate_hz=20.0, clients=64):
    """The seeded 64-episode mixed batch (grids 401x201 .. 2001x1001, 1-4
    wings): (1) every episode advanced `steps` steps, all resident and in
    flight at once (FP32; packed launches over all episodes, and each episode
    on its own streams), against the same episodes served one at a time
    through the plain FP64 path; (2) 64 online clients (one per episode) on
    the ZeroMQ server with Poisson arrivals, segments of 100-2000 steps, SAVE
    with p = 0.05: STEP latency percentiles at the client; (3) the FP32
    path's segment-averaged forces against FP64 for one client's segments."""
    from lbm_mutiwing_b200 import api, batch, loadgen
    from lbm_mutiwing_b200 import protocol as P
    from lbm_mutiwing_b200 import workloads as wl
    eps = wl.mixed_batch(64, steps=2 * steps + 16)
    nodes = sum(e.nx * e.ny for e in eps)
    sims = batch.create(eps, api.PRECISION_FP32)
    packed = api.Batch(0)
    batch.advance_packed(sims, 4, first_cycle=1, packed=packed)
    wall = batch.advance_packed(sims, steps, first_cycle=5, packed=packed)
    packed.close()
    batched = nodes * steps / wall / 1e6
    batch.advance_together(sims, 4, first_cycle=steps + 5)
    wall_streams = batch.advance_together(sims, steps, first_cycle=steps + 9)
    for s in sims:
        s.close()
    batched_streams = nodes * steps / wall_streams / 1e6
    plain_s, plain_nu = batch.advance_one_at_a_time(eps, max(8, steps // 4))
    plain = plain_nu / plain_s / 1e6
    served = served_metrics(clients, requests, rate_hz)
    # FP32 vs FP64 segment-averaged forces of one client's segments
    ep = wl.by_name("mix:1")
    rng = np.random.default_rng(7)
    dt = ep.scale * ep.uu
    lines, cyc = ["RESET 0.0"], 1
    for n in (150, 400, 250):
        cyc += n
        lines.append(loadgen.step_line((cyc - 1) * dt, rng.normal(0, 0.05, 3 * ep.wing_count)))
    from lbm_mutiwing_b200.session import EpisodeSession
    rows = {}
    for prec in (api.PRECISION_FP64, api.PRECISION_FP32):
        with api.Simulation(ep, prec, motion_source=api.MOTION_STREAM) as sim:
            se = EpisodeSession(sim, ep)
            rows[prec] = [np.array(P.parse_force_reply(se.handle(P.parse(l, ep.wing_count)))) for l in lines]
    W = ep.wing_count
    err = 0.0
    for a, b in zip(rows[api.PRECISION_FP32], rows[api.PRECISION_FP64]):
        fa, fb = a[1:1 + 3 * W], b[1:1 + 3 * W]
        err = max(err, float(np.max(np.abs(fa - fb)) / max(float(np.max(np.abs(fb))), 1e-30)))
    return {"episodes": len(eps), "nodes": nodes, "wings": sum(e.wing_count for e in eps),
            "wings_drawn": sum(e.meta.get("wings_drawn", e.wing_count) for e in eps),
            "heave_draws_capped": sum(e.meta.get("heave_capped", 0) for e in eps),
            "draw_caps": "wing count capped by what the domain holds (wings 1.5 chords apart); heave amplitude "
                         "capped at 0.3 h - 0.5 chords so wings stay clear of the borders",
            "batched_fp32_mlups": batched, "batched_streams_fp32_mlups": batched_streams,
            "one_at_a_time_fp64_mlups": plain,
            "batched_over_one_at_a_time": batched / plain,
            "batched_over_streams_fp32": batched / batched_streams,
            **served,
            "fp32_vs_fp64_force_max_rel_err": err,
            "force_err_sample": "segment-averaged per-wing Fx, Fy, M of mix episode 1, 3 STEP segments"}


def served_metrics(clients=64, requests=3, rate_hz=20.0):
    """`clients` online clients on the ZeroMQ server (client k runs mixed
    episode k mod 64), Poisson arrivals at rate_hz per client, segments of
    100-2000 steps, SAVE with p = 0.05: STEP latency at the client.  The
    server admits episodes by free device memory."""
    import threading
    from lbm_mutiwing_b200 import api, loadgen
    from lbm_mutiwing_b200 import workloads as wl
    from lbm_mutiwing_b200.serve import Server
    srv = Server("tcp://127.0.0.1:0", wl.by_name, "mix:0", precision=api.PRECISION_FP32, workers=clients)
    th = threading.Thread(target=srv.serve, kwargs={"idle_timeout_s": 600}, daemon=True)
    th.start()
    names = [f"mix:{k % 64}" for k in range(clients)]
    res = loadgen.poisson_load(f"tcp://127.0.0.1:{srv.port}", names, wl.by_name, requests_per_client=requests,
                               rate_hz=rate_hz)
    srv.stop()
    th.join(60)
    srv.close()
    return {"served_clients": clients, "served_rate_hz_per_client": rate_hz, "served_steps": len(res.step_latency_s),
            "served_step_p50_ms": res.percentile(50) * 1e3, "served_step_p99_ms": res.percentile(99) * 1e3,
            "served_mlups": res.mlups(), "served_errors": len(res.errors)}


def sharded_batch(ranks, steps, warmup, rank, world, local):
    """The 64-episode mixed batch split over the ranks (each rank one packed
    engine on its GPU): whole-job MLUPS = all node updates / slowest rank."""
    from lbm_mutiwing_b200 import batch
    from lbm_mutiwing_b200 import workloads as wl
    eps = wl.mixed_batch(64, steps=steps + warmup + 8)
    mine, nu, sec = batch.sharded_packed_run(eps, steps, warmup, rank, world,
                                             engine=batch.PackedEngine(local), barrier=ranks.barrier)
    smax = ranks.allmax(sec)
    total = sum(e.nx * e.ny for e in eps) * steps
    return {"episodes": len(eps), "episodes_this_rank": len(mine), "steps": steps,
            "mlups": total / smax / 1e6, "seconds_max": smax,
            "timing": "wall clock around the synchronous packed call, max over ranks"}


def run_ours(args):
    from lbm_mutiwing_b200 import ranks
    rank, world, local = ranks.init("nccl")
    import torch
    from lbm_mutiwing_b200 import api, build
    if rank == 0:
        build.build()
    ranks.barrier()
    torch.cuda.set_device(local)
    prec = api.PRECISION_FP32 if args.precision == "fp32" else api.PRECISION_FP64
    K, Wm = args.steps, max(3, args.warmup)
    max_reps = max(3, MAX_TIMED_STEPS // max(K, 1))
    KP = min(K, 100)
    ep = workload(args.workload, Wm + max_reps * K + KP + 8)
    nodes = ep.nx * ep.ny
    tiles = {"auto": 0, "short": api.FLAG_PASS_SHORT_TILES, "tall": api.FLAG_PASS_TALL_TILES}[args.pass_tiles]
    sim = api.Simulation(ep, prec, device=local, flags=tiles)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    # warm-up (builds the step graphs)
    sim.step(Wm, first_cycle=1, rows=False)
    torch.cuda.synchronize()
    # timed region: K steps per repetition, device time by CUDA events on the
    # library stream; repetitions back to back for CLOCK_WINDOW_S seconds
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = []
    cyc = Wm + 1
    with Clocks(local) as clk:
        clk.begin()
        t_start = time.perf_counter()
        while True:
            ranks.barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            sim.step(K, first_cycle=cyc, rows=False)
            e1.record(stream)
            torch.cuda.synchronize()
            reps.append(e0.elapsed_time(e1))
            cyc += K
            elapsed = ranks.allmax(time.perf_counter() - t_start)
            if len(reps) >= max_reps or (len(reps) >= 3 and elapsed >= CLOCK_WINDOW_S):
                break
        clk.end()
    reps_max = [ranks.allmax(r) for r in reps]
    ms = statistics.median(reps_max)
    # phase breakdown and the bulk kernel's launch time: a second pass with
    # CUDA events around every phase (kernels launched directly)
    sim.set_timing(True)
    sim.step(KP, first_cycle=cyc, rows=False)
    phases = sim.phase_times()
    sim.set_timing(False)
    ranks.barrier()
    value = ranks.whole_job_rate(nodes * K, world, ms / 1e3) / 1e6
    sim.close()

    # the plain FP64 path on the same workload (the drop-in), events on its stream
    plain = None
    if prec == api.PRECISION_FP32:
        KF = min(K, 40)
        s64 = api.Simulation(ep, api.PRECISION_FP64, device=local)
        st64 = torch.cuda.ExternalStream(s64.stream(), device=local)
        s64.step(3, first_cycle=1, rows=False)
        ranks.barrier()
        torch.cuda.synchronize()
        e0.record(st64)
        s64.step(KF, first_cycle=4, rows=False)
        e1.record(st64)
        torch.cuda.synchronize()
        ms64 = ranks.allmax(e0.elapsed_time(e1))
        s64.close()
        mlups64 = ranks.whole_job_rate(nodes * KF, world, ms64 / 1e3) / 1e6
        plain = {"mlups": mlups64, "ms_per_step": ms64 / KF, "steps": KF, "fp32_over_fp64": value / mlups64}

    # e2e: online STEP segments (driver.f90:174-195) through the C ABI with
    # host buffers -- per segment the start and target motion rows go to the
    # device, and every step's force row comes back.
    sim_e = api.Simulation(ep, prec, motion_source=api.MOTION_STREAM, device=local, flags=tiles)
    ncol = 1 + 9 * ep.wing_count
    # online rows carry displacements relative to the wing bases (mode.f90:207-214)
    motion_rows = ep.motion.copy()
    for w in range(ep.wing_count):
        motion_rows[:, 4 + 9 * w] -= ep.wing_x_origin + w * ep.wing_x_spacing
        motion_rows[:, 7 + 9 * w] -= ep.wing_y_origin
    sim_e.set_stream_rows(motion_rows[0], motion_rows[SEG])
    sim_e.step(Wm, first_cycle=1, rows=False)
    ranks.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done, cyc = 0, Wm + 1
    while done < K:
        n = min(SEG, K - done)
        a = motion_rows[cyc - 1]
        b = motion_rows[min(cyc - 1 + n, motion_rows.shape[0] - 1)]
        sim_e.set_stream_rows(a, b)
        out = sim_e.step(n, first_cycle=cyc, rows=True)
        assert out.shape == (n, sim_e.row_len)
        done += n
        cyc += n
    torch.cuda.synchronize()
    e2e_s = ranks.allmax(time.perf_counter() - t0)
    e2e = ranks.whole_job_rate(nodes * K, world, e2e_s) / 1e6
    h2d = 2 * ncol * 8 / SEG
    d2h = sim_e.row_len * 8
    sim_e.close()

    # roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    interior = (ep.nx - 2) * (ep.ny - 2)
    if prec == api.PRECISION_FP32 and phases.get("passes", 0) > 0:
        kernel = "pass_far_kernel"
        launches = phases["passes"]
        kernel_ms = phases["pass_far_ms"] / launches
        alg_bytes = 72 * phases["far_tile_nodes"] / launches
        step_bytes = 36 * interior
    else:
        kernel = "fused_bulk_tma_kernel" if prec == api.PRECISION_FP32 else "plain stream+moments+collide"
        kernel_ms = phases["collide_stream_ms"] / max(1, phases["steps"])
        alg_bytes = (72 if prec == api.PRECISION_FP32 else 144) * interior
        step_bytes = alg_bytes
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    roof = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": ncu_traffic(ep.name, kernel) if prec == api.PRECISION_FP32 else None,
            "algorithmic_bytes_per_launch": alg_bytes, "mean_launch_ms": kernel_ms,
            "whole_step_frac": step_bytes * K / (ms / 1e3) / 1e9 / peak,
            "one_step_equivalent_frac": (72 if prec == api.PRECISION_FP32 else 144) * interior * K
                                        / (ms / 1e3) / 1e9 / peak}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": Wm,
            "ms_per_step": ms / K, "timed_repeats": len(reps),
            "ms_per_step_min_max": [min(reps_max) / K, max(reps_max) / K],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == api.PRECISION_FP32 else "f64",
            "data": "synthetic (seeded NACA0012 geometry, analytic pitch/heave motion)",
            "config": config_of(ep, "fp32 deviation" if prec == api.PRECISION_FP32 else "fp64 plain", world),
            "phases_ms_per_step": {k: v / max(1, phases["steps"]) for k, v in phases.items()
                                   if k != "steps"},
            "roofline": roof,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "segment_steps": SEG},
            "clocks": clk.summary(),
            "gpu_launches": len(reps) * kernels_in_call(K, args.precision)}
    if prec == api.PRECISION_FP32 and roof["kernel"] == "pass_far_kernel":
        tall = args.pass_tiles == "tall" or (args.pass_tiles == "auto" and nodes >= 32 << 20)
        roof["tile"] = "64x12" if tall else "64x8"   # the far-tile kernel's tile (nodes)
    if plain:
        line["plain_fp64"] = plain
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["parity"], line["cpu_baseline"] = parity_and_cpu_baseline(args.workload)
    if not args.no_serving:
        if world == 1:
            line["serving"] = serving_metrics()
        else:
            line["batched_sharded"] = sharded_batch(ranks, 200, 8, rank, world, local)
    if rank == 0:
        print(json.dumps(line))
    ranks.finish()


def run_packed(args):
    """The seeded 64-episode mixed batch, every kernel of a step one launch
    over the episodes of this rank's shard: W warm-up steps (long enough,
    from 8, to let the engine tune its bulk kernel), then K timed steps (wall
    clock around the synchronous call, max over ranks)."""
    from lbm_mutiwing_b200 import build, ranks
    from lbm_mutiwing_b200 import workloads as wl
    rank, world, local = ranks.init("nccl")
    if rank == 0:
        build.build()
    ranks.barrier()
    K, Wm = args.steps, max(3, args.warmup)
    res = sharded_batch(ranks, K, Wm, rank, world, local)
    eps = wl.mixed_batch(64, steps=8)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": res["mlups"], "unit": UNIT, "n_gpus": world, "steps": K,
                          "warmup": Wm, "ms_per_step": res["seconds_max"] / K * 1e3, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": "mixed64_packed", "episodes": len(eps),
                                     "nodes": sum(e.nx * e.ny for e in eps),
                                     "wings": sum(e.wing_count for e in eps), "markers": MARKERS,
                                     "parallelism": f"64 episodes split over {world} GPUs"}}))
    ranks.finish()


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(argv, args.gpus)
    if args.impl == "reference":
        run_reference(args)
    elif args.packed:
        run_packed(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
