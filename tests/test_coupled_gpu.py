"""Wings whose supports share lattice nodes, through the C ABI, against the
oracle's one dense system over all segments (boundary_condition.f90:
1609-1640).

* Two NACA0012 sections in tandem with the trailing edge of the first 1.5-2
  lattice spacings from the leading edge of the second: their 6 x 6 support
  boxes share 17-18 nodes, G couples the wings, and the library solves the joint
  system (conjugate gradients preconditioned by the per-wing factors).
  Tolerances as for well-conditioned single wings: FP64 path 1e-9 relative
  on segment-averaged forces and on u, v; FP32 path 1e-3 on forces.
* A staggered pair whose bounding boxes overlap but whose supports do not
  touch: no coupling is reported.
"""
import math

import numpy as np
import pytest

from lbm_mutiwing_b200 import api
from lbm_mutiwing_b200 import workloads as wl

pytestmark = pytest.mark.gpu

COUPLED = 16
NOCONV = 32


def coupled_episode(steps=40):
    # chord 50 nodes, 100 markers at equal arc length (about one spacing
    # apart); axes 1.03 chords apart, same phase, pitch 3 deg: the gap
    # between the sections stays 1.5-2 spacings
    return wl.tandem_pitch_heave("coupled", 5.0, 2.5, 0.02, 100.0, -1.0, 0.0, 100, steps, n_wings=2,
                                 x_spacing=1.03, lag=0.0, pitch_deg=3.0, heave=0.1, freq=1.0)


def staggered_episode(steps=10):
    nx, ny, ox, oy = wl.lattice(5.0, 2.5, 0.02)
    ep = wl.Episode(name="staggered", nx=nx, ny=ny, scale=0.02, re=100.0, ox=ox, oy=oy,
                    wing_x_origin=-1.0, wing_x_spacing=0.9, wing_y_origin=0.0, steps=steps)
    ep.markers = [wl.naca_loop(0.12, 100), wl.naca_loop(0.12, 100)]
    wings = [wl.WingMotion(x=-1.0, y=0.0, pitch_amp=0.0, heave_amp=0.0),
             wl.WingMotion(x=-0.1, y=0.2, pitch_amp=0.0, heave_amp=0.0)]
    dt = ep.scale * ep.uu
    ep.motion = wl.motion_table(wings, (steps + 1) * dt, dt)
    return ep


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_coupled_wings_solved_jointly(gpu_lib, oracle_lib):
    from oracle import fields as F
    ep = coupled_episode(40)
    o = oracle_lib.Oracle(ep)
    ro = o.run(1, 40)
    u_o, v_o = o.field("u"), o.field("v")
    with api.Simulation(ep, api.PRECISION_FP64) as s:
        r64 = s.step(40)
        _, u64, v64, _ = s.fields()
        res = s.ibm_residual()
        st = s.status()
    assert st & COUPLED and not st & NOCONV, st
    assert res < 1e-10, res
    e64 = F.force_error(F.segment_average(r64, 2), F.segment_average(ro, 2))
    assert e64 <= 1e-9, e64
    assert rel(u64, u_o) <= 1e-9 and rel(v64, v_o) <= 1e-9, (rel(u64, u_o), rel(v64, v_o))
    with api.Simulation(ep, api.PRECISION_FP32) as s:
        r32 = s.step(40, flags=api.STEP_FIELDS)
        st32 = s.status()
    assert st32 & COUPLED and not st32 & NOCONV, st32
    e32 = F.force_error(F.segment_average(r32, 2), F.segment_average(ro, 2))
    assert e32 <= 1e-3, e32
    print(f"\ncoupled wings: fp64 force {e64:.2e}, u {rel(u64, u_o):.2e}, residual {res:.2e}; fp32 force {e32:.2e}")


def test_coupled_wings_packed_equal_alone(gpu_lib):
    """The joint solve in packed launches (one episode coupled, one not)
    gives the same bits as each episode stepped alone."""
    eps = [coupled_episode(20), staggered_episode(20)]
    alone = []
    for ep in eps:
        with api.Simulation(ep, api.PRECISION_FP32) as s:
            alone.append((s.step(20), s.f()))
    sims = [api.Simulation(ep, api.PRECISION_FP32) for ep in eps]
    try:
        with api.Batch(0) as b:
            rows = b.step(sims, 20)
        for (ra, fa), rb, s in zip(alone, rows, sims):
            assert np.array_equal(ra, rb)
            assert np.array_equal(fa, s.f())
    finally:
        for s in sims:
            s.close()


def test_staggered_wings_apart_are_not_coupled(gpu_lib, oracle_lib):
    ep = staggered_episode(10)
    o = oracle_lib.Oracle(ep)
    ro = o.run(1, 10)
    with api.Simulation(ep, api.PRECISION_FP64) as s:
        r = s.step(10)
        assert s.status() & COUPLED == 0
        assert s.ibm_residual() < 1e-10
    assert rel(r[:, 1:7], ro[:, 1:7]) < 1e-9
    assert math.isfinite(float(np.abs(r).max()))
