"""Known-answer tests that pin the CPU oracle (no GPU needed).

The reference ships no golden vectors, so the oracle is pinned by properties
its equations must satisfy and by its own committed regression fixture
(tests/golden/oracle_regression.json, made by tests/golden/make_golden.py).
"""
import json
import math
import os

import numpy as np
import pytest

from lbm_mutiwing_b200 import workloads as wl

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

M = np.array([[1, 1, 1, 1, 1, 1, 1, 1, 1], [-4, -1, -1, -1, -1, 2, 2, 2, 2],
              [4, -2, -2, -2, -2, 1, 1, 1, 1], [0, 1, 0, -1, 0, 1, -1, -1, 1],
              [0, -2, 0, 2, 0, 1, -1, -1, 1], [0, 0, 1, 0, -1, 1, 1, -1, -1],
              [0, 0, -2, 0, 2, 1, 1, -1, -1], [0, 1, -1, 1, -1, 0, 0, 0, 0],
              [0, 0, 0, 0, 0, 1, -1, 1, -1]], dtype=float)


def small_episode(wings=1, scale=0.02, width=4.0, height=2.0, markers=60, spacing="uniform",
                  steps=40, re=100.0, pitch=10.0, heave=0.2):
    return wl.tandem_pitch_heave("kat", width, height, scale, re, -0.75, 0.0, markers, steps,
                                 n_wings=wings, spacing=spacing, pitch_deg=pitch, heave=heave,
                                 x_spacing=1.5)


def test_mrt_inverse(oracle_lib):
    minv = oracle_lib.inverse_m()
    assert np.abs(M @ minv - np.eye(9)).max() < 1e-15
    exact = M.T / np.diag(M @ M.T)[None, :]
    assert np.abs(minv - exact).max() < 1e-15


def test_delta_kernel_partition_of_unity(oracle_lib):
    for r in np.linspace(0.0, 1.0, 37):
        s = sum(oracle_lib.delta_phi(r - k) for k in range(-3, 4))
        assert abs(s - 1.0) < 1e-12, r
    # compact support of 2.5 spacings and symmetry
    assert oracle_lib.delta_phi(2.5000001) == 0.0
    assert abs(oracle_lib.delta_phi(2.5)) < 1e-15
    assert oracle_lib.delta_phi(0.7) == oracle_lib.delta_phi(-0.7)


def test_motion_ramp_endpoints(oracle_lib):
    s0, v0, v1, dt = 0.3, 0.1, 0.5, 0.2
    s, v, a = oracle_lib.interpolate_triplet(s0, v0, v1, dt, 0.0)
    assert (s, v) == (s0, v0) and a == 0.0
    s, v, a = oracle_lib.interpolate_triplet(s0, v0, v1, dt, dt)
    assert abs(v - v1) < 1e-15 and abs(a) < 1e-12
    assert abs(s - (s0 + dt * (v0 + v1) / 2)) < 1e-15
    # degenerate segment (mode.f90:275-280)
    s, v, a = oracle_lib.interpolate_triplet(s0, v0, v1, 0.0, 0.1)
    assert (v, a) == (v1, 0.0) and abs(s - (v1 * 0.1 + s0)) < 1e-15


def test_uniform_flow_interior_invariant(oracle_lib):
    ep = wl.Episode(name="empty", nx=41, ny=21, scale=0.05, re=100.0, ox=-1.0, oy=-0.5)
    o = oracle_lib.Oracle(ep)
    f_init = o.f()
    n = 5
    for c in range(1, n + 1):
        o.step(c)
    f = o.f()
    inner = (slice(None), slice(n + 1, -n - 1), slice(n + 1, -n - 1))
    # feq with single-precision weights is an MRT fixed point up to rounding of w
    assert np.abs(f[inner] - f_init[inner]).max() < 1e-9
    # the walls (u = v = 0 rows) disturb the flow next to them
    assert np.abs(f[:, 1, :] - f_init[:, 1, :]).max() > 1e-6


def test_collision_conserves_mass_and_momentum(oracle_lib):
    ep = wl.Episode(name="empty", nx=21, ny=21, scale=0.05, re=100.0, ox=-0.5, oy=-0.5)
    o = oracle_lib.Oracle(ep)
    rng = np.random.default_rng(1)
    f = o.f() * (1.0 + 0.01 * rng.standard_normal((9, 21, 21)))
    o.set_f(f)
    o.step(1)
    f0 = o.f0()        # post-stream, pre-collision
    f1 = o.f()         # post-collision (interior)
    ex = M[3]
    ey = M[5]
    sl = (slice(None), slice(1, -1), slice(1, -1))
    for mom in (M[0], ex, ey):
        a = np.tensordot(mom, f0[sl], 1)
        b = np.tensordot(mom, f1[sl], 1)
        assert np.abs(a - b).max() < 1e-14


def test_band_rule(oracle_lib):
    ep = small_episode()
    o = oracle_lib.Oracle(ep)
    o.step(1)
    band = o.band()
    _, _, xb2, yb2 = o.markers()
    # recompute the first-claimant list of airfoil.f90:286-335 in Python
    expect, seen = [], set()
    for s in range(len(xb2)):
        xs = ep.ox + ep.scale * np.arange(ep.nx)
        ys = ep.oy + ep.scale * np.arange(ep.ny)
        ii = [i for i in range(ep.nx) if abs((xs[i] - xb2[s]) / ep.scale) <= 2.5]
        jj = [j for j in range(ep.ny) if abs((ys[j] - yb2[s]) / ep.scale) <= 2.5]
        assert len(ii) <= 6 and len(jj) <= 6
        for i in ii:
            for j in jj:
                if (i, j) not in seen:
                    seen.add((i, j))
                    expect.append((i + 1, j + 1, 1))
    assert [tuple(r) for r in band] == expect


def test_ibm_no_slip_residual(oracle_lib):
    o = oracle_lib.Oracle(small_episode())
    for c in range(1, 4):
        o.step(c)
        assert o.ibm_residual() < 1e-9


def test_symmetric_section_zero_lift(oracle_lib):
    ep = small_episode(pitch=0.0, heave=0.0)
    ep.motion[:, 7] = 0.0   # y column of wing 1: on the lattice's axis of symmetry
    ep.wing_y_origin = 0.0
    o = oracle_lib.Oracle(ep)
    rows = o.run(1, 20)
    fx, fy = rows[:, 1], rows[:, 2]
    assert np.all(np.abs(fy) < 1e-9 * np.abs(fx).max())


def test_motion_table_lookup(oracle_lib):
    ep = small_episode(steps=10)
    o = oracle_lib.Oracle(ep)
    rows = o.run(1, 10)
    # force-row motion columns echo the table (x, xv, xa, y, yv, ya, angle, omega, omgac)
    for n in range(10):
        tab = ep.motion[n]
        got = rows[n, 1 + 3 + 3:1 + 3 + 3 + 9]
        want = np.array([tab[4], tab[5], tab[6], tab[7], tab[8], tab[9], tab[1], tab[2], tab[3]])
        assert np.allclose(got, want, rtol=0, atol=1e-12)
        assert abs(rows[n, 0] - n * ep.scale * ep.uu) < 1e-15


def test_stream_rows_match_triplets(oracle_lib):
    ep = small_episode(steps=10)
    o = oracle_lib.Oracle(ep, motion_source=2)
    start = np.zeros(10)
    start[1:10] = [0.1, 0.2, 0.0, 0.5, 0.3, 0.0, 0.05, -0.1, 0.0]
    target = o.build_stream_target_row(start, 0.01, np.array([0.01, 0.4, -0.2, 0.3]))
    o.set_stream_rows(start, target)
    mid = o.stream_row(0.005)
    s, v, a = oracle_lib.interpolate_triplet(0.1, 0.2, 0.6, 0.01, 0.005)
    assert np.allclose(mid[1:4], [s, v, a], atol=1e-15)
    assert np.allclose(o.stream_row(-1.0)[1:], start[1:])


def test_regression_fixture(oracle_lib):
    """The oracle reproduces its committed regression run bit for bit."""
    with open(os.path.join(GOLDEN, "oracle_regression.json")) as fh:
        gold = json.load(fh)
    from tests.golden.make_golden import run_case
    got = run_case(oracle_lib)
    assert got["band_n"] == gold["band_n"]
    assert np.array_equal(np.array(got["rows"]), np.array(gold["rows"]))
    for k in ("f_sum", "u_sum", "v_sum"):
        assert got[k] == gold[k], k
