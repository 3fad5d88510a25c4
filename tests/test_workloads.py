import math

import numpy as np

from lbm_mutiwing_b200 import workloads as wl


def test_naca_loop_layout():
    pts = wl.naca_loop(0.12, 200)
    assert pts.shape == (201, 2)
    assert np.array_equal(pts[0], pts[-1])
    assert abs(pts[0, 0] + 0.25) < 1e-15 and pts[0, 1] == 0.0
    assert abs(pts[100, 0] - 0.75) < 1e-15 and abs(pts[100, 1]) < 1e-15
    assert np.all(pts[1:100, 1] > 0) and np.all(pts[101:200, 1] < 0)
    # 12 % thickness
    assert abs(2 * pts[:, 1].max() - 0.12) < 2e-3


def test_reference_geometry_file_matches_layout():
    import os
    p = os.path.join(os.path.dirname(__file__), "golden", "boundary.dat")
    pts = wl.read_boundary_file(p)
    assert pts.shape == (205, 2)
    assert np.array_equal(pts[0], pts[-1])
    assert abs(pts[:, 0].min() + 0.25) < 1e-8 and abs(pts[:, 0].max() - 0.75) < 1e-8


def test_tandem_800x400_geometry():
    ep = wl.tandem_800x400(steps=10)
    assert (ep.nx, ep.ny) == (801, 401)
    assert (ep.ox, ep.oy) == (-4.0, -2.0)
    assert ep.wing_count == 2 and ep.markers[0].shape == (201, 2)
    assert ep.motion.shape[1] == 19
    # pitch 15 deg sin(2 pi f t), f = 0.5, wing 2 lags pi/4
    t = ep.motion[:, 0]
    assert np.allclose(ep.motion[:, 1], 15 * math.pi / 180 * np.sin(math.pi * t))
    assert np.allclose(ep.motion[:, 10], 15 * math.pi / 180 * np.sin(math.pi * t - math.pi / 4))
    assert np.allclose(ep.motion[:, 4], -2.0) and np.allclose(ep.motion[:, 13], -0.5)


def test_mixed_batch_is_seeded():
    a = wl.mixed_batch(8, seed=5, steps=10)
    b = wl.mixed_batch(8, seed=5, steps=10)
    assert [e.nx for e in a] == [e.nx for e in b]
    assert all(np.array_equal(x.motion, y.motion) for x, y in zip(a, b))
    assert {e.nx for e in wl.mixed_batch(64, steps=2)} <= {401, 801, 1201, 2001}


def test_arc_spacing_is_even_and_closed():
    # the default marker spacing: equal arc length along each surface
    pts = wl.naca_loop(0.12, 200)
    seg = np.hypot(*np.diff(pts * 100.0, axis=0).T)   # chord of 100 lattice spacings
    assert 1.0 <= seg.min() and seg.max() <= 1.03
    assert np.array_equal(pts[0], pts[-1])
    assert abs(pts[100, 0] - 0.75) < 1e-15 and abs(pts[100, 1]) < 1e-15
    cos = np.hypot(*np.diff(wl.naca_loop(0.12, 200, "cosine") * 100.0, axis=0).T)
    assert cos.min() < 0.03   # what the arc spacing avoids
