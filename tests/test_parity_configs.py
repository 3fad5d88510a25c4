"""GPU parity on the benchmark configurations, through the C ABI, against the
CPU FP64 oracle run on the same seeded inputs in the same process.

Cases:
  * the 800x400 two-wing tandem (801 x 401 nodes, Re 200, two NACA0012 wings
    of 200 markers each, pitch 15 deg and heave 0.5 chord at f = 0.5 with a
    pi/4 lag), the full 2000 steps;
  * a 60-step window from the start of the 4000x2000 tandem (4001 x 2001
    nodes, Re 1000);
  * a reduced-size regression driven by the reference's own offline motion
    table: a 400-step window of motion_params.dat (tests/golden/
    motion_params_window.dat, rows from t = 2.25 with the time re-based) on
    two wings of the reference's own marker file boundary.dat, on an 8 x 4
    chord lattice at dx = 0.01.

Markers of the synthetic NACA sections sit at equal arc length along each
surface (1.0-1.02 lattice spacings apart at 200 markers on a 100-node
chord); the configurations' cosine spacing puts trailing-edge markers 0.025
spacings apart, where the immersed-boundary system is singular and the FP64
oracle itself diverges after about 1150 steps of the 800x400 case.

Every case reports, per path: the relative L2 error of u, v, p and vorticity
(solution.f90:185-205) after the last step, and the largest relative error
of the segment-averaged per-wing Fx, Fy and M (the FORCE reply average of
driver.f90:260-289) over consecutive segments of the run.

Tolerances, written per case below:
  * plain FP64 path: forces 1e-9 relative (the banded LDL^T solve in RCM
    order against the oracle's dense partial-pivot LU on well-conditioned
    marker sets), fields 1e-9 relative L2;
  * fused FP32 path: forces 1e-3 relative (the accuracy the FP32 deviation
    storage is built to), u, v and vorticity 2e-3, p 1e-6 relative L2.
"""
import os
import threading

import numpy as np
import pytest

from lbm_mutiwing_b200 import api
from lbm_mutiwing_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

FP64_FORCE, FP64_FIELD = 1e-9, 1e-9
FP32_FORCE, FP32_UV, FP32_P = 1e-3, 2e-3, 1e-6


def oracle_run(oracle_lib, ep, steps, out):
    """The oracle on all host cores (run in a thread beside the GPU)."""
    o = oracle_lib.Oracle(ep, nthreads=os.cpu_count() or 1)
    out["rows"] = o.run(1, steps)
    out["u"], out["v"], out["p"] = o.field("u"), o.field("v"), o.field("pre")
    o.close()


def gpu_run(ep, precision, steps):
    with api.Simulation(ep, precision) as s:
        rows = s.step(steps, flags=api.STEP_FIELDS)
        _, u, v, p = s.fields()
        assert s.status() & ~8 == 0
    return rows, u, v, p


def compare(ep, steps, segment, oracle_lib):
    from oracle import fields as F
    ref = {}
    th = threading.Thread(target=oracle_run, args=(oracle_lib, ep, steps, ref))
    th.start()
    got = {prec: gpu_run(ep, prec, steps) for prec in (api.PRECISION_FP64, api.PRECISION_FP32)}
    th.join()
    W = ep.wing_count
    report = {}
    for prec, (rows, u, v, p) in got.items():
        ferr = 0.0
        for a in range(0, steps, segment):
            ferr = max(ferr, F.force_error(F.segment_average(rows[a:a + segment], W),
                                           F.segment_average(ref["rows"][a:a + segment], W)))
        e = F.field_errors(u, v, p, ref["u"], ref["v"], ref["p"], ep.uu, ep.scale)
        e["force_max_rel"] = ferr
        report["fp64" if prec == api.PRECISION_FP64 else "fp32"] = e
        # motion columns follow the same table lookup
        assert np.allclose(rows[:, 4 + 3 * W:], ref["rows"][:, 4 + 3 * W:], rtol=1e-13, atol=1e-15)
    print(f"\nparity {ep.name} ({ep.nx}x{ep.ny}, {steps} steps, segments of {segment}): {report}")
    return report


def check(report):
    e64, e32 = report["fp64"], report["fp32"]
    assert e64["force_max_rel"] <= FP64_FORCE, e64
    for k in ("u_l2", "v_l2", "p_l2", "vort_l2"):
        assert e64[k] <= FP64_FIELD, (k, e64)
    assert e32["force_max_rel"] <= FP32_FORCE, e32
    for k in ("u_l2", "v_l2", "vort_l2"):
        assert e32[k] <= FP32_UV, (k, e32)
    assert e32["p_l2"] <= FP32_P, e32


def test_tandem_800x400_full_run(gpu_lib, oracle_lib):
    ep = wl.tandem_800x400(steps=2000)
    check(compare(ep, 2000, 500, oracle_lib))


def test_tandem_4000x2000_window(gpu_lib, oracle_lib):
    ep = wl.tandem_4000x2000(steps=60)
    check(compare(ep, 60, 20, oracle_lib))


def reference_motion_episode(steps=400):
    """Two wings of the reference's boundary.dat on an 8 x 4 chord lattice at
    dx = 0.01 (dt = 1e-4, one motion row per step), driven by the window of
    the reference's motion_params.dat (absolute x = 0 / 1.5, y about 0)."""
    pts = wl.read_boundary_file(os.path.join(GOLDEN, "boundary.dat"))
    rows = wl.read_motion_file(os.path.join(GOLDEN, "motion_params_window.dat"), 2)
    nx, ny, ox, oy = wl.lattice(8.0, 4.0, 0.01)
    ep = wl.Episode(name="reference_motion_800x400", nx=nx, ny=ny, scale=0.01, re=500.0, ox=ox, oy=oy,
                    wing_x_origin=0.0, wing_x_spacing=1.5, wing_y_origin=0.5, steps=steps)
    ep.markers = [pts, pts.copy()]
    ep.motion = rows
    return ep


def test_reference_motion_table_regression(gpu_lib, oracle_lib):
    ep = reference_motion_episode(400)
    check(compare(ep, 400, 100, oracle_lib))
