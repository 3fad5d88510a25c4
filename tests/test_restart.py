"""Restart files in the reference's layout (saveflowfield / readflowfield,
solution.f90:1616-1851): the byte layout against an independent reader, the
encode / decode round trip, and (GPU) a run continued from a file against
the same run continued in memory."""
import os
import struct

import numpy as np
import pytest

from lbm_mutiwing_b200 import restart


def _sample(nx=7, ny=5, W=2, seed=3):
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(ny, nx))
    v = rng.normal(size=(ny, nx))
    f = rng.normal(size=(9, ny, nx))
    border = rng.normal(size=(9, 2 * ny + 2 * nx))
    left, right, bottom, top = restart._border_layout(nx, ny)
    # the two copies of each corner node agree, as the library keeps them
    border[:, left[0]] = border[:, bottom[0]]
    border[:, left[ny - 1]] = border[:, top[0]]
    border[:, right[0]] = border[:, bottom[nx - 1]]
    border[:, right[ny - 1]] = border[:, top[nx - 1]]
    return u, v, f, border


def test_layout_matches_reference_record_order():
    nx, ny, W = 7, 5, 2
    u, v, f, border = _sample(nx, ny, W)
    data = restart.encode(123, W, -1, u, v, f, border, 0.01)
    assert len(data) == 4 + 4 + 8 * 11 * W + 4 + 8 * 11 * nx * ny + 8 * 36 * (ny - 2) + 8 * 36 * nx
    cycle, wc = struct.unpack_from("<ii", data, 0)
    assert (cycle, wc) == (123, W)
    o = 8 + 88 * W
    assert struct.unpack_from("<i", data, o)[0] == -1
    o += 4
    # node (i, j) = (3, 2) (1-based): record (j - 1) * nx + (i - 1): u, v, f(1:9)
    rec = struct.unpack_from("<11d", data, o + 88 * (1 * nx + 2))
    assert rec[0] == u[1, 2] and rec[1] == v[1, 2]
    assert list(rec[2:]) == list(f[:, 1, 2])
    # column record of j = 3: leftf2, f0(1, j), rightf2, f0(Nx, j)
    o_cols = o + 88 * nx * ny
    colrec = struct.unpack_from("<36d", data, o_cols + 288 * 1)
    feq = restart.initial_equilibrium(0.01)
    left, right, bottom, top = restart._border_layout(nx, ny)
    assert np.array_equal(colrec[0:9], feq) and np.array_equal(colrec[18:27], feq)
    assert list(colrec[9:18]) == list(border[:, left[2]])
    assert list(colrec[27:36]) == list(border[:, right[2]])
    # row record of i = 4: upf2, f0(i, Ny), downf2, f0(i, 1)
    rowrec = struct.unpack_from("<36d", data, o_cols + 288 * (ny - 2) + 288 * 3)
    assert list(rowrec[9:18]) == list(border[:, top[3]])
    assert list(rowrec[27:36]) == list(border[:, bottom[3]])


def test_round_trip_and_refusals():
    nx, ny, W = 7, 5, 2
    u, v, f, border = _sample(nx, ny, W)
    data = restart.encode(77, W, 2, u, v, f, border, 0.01)
    cycle, movenum, u2, v2, f2, b2 = restart.decode(data, nx, ny, W)
    assert (cycle, movenum) == (77, 2)
    for a, b in ((u, u2), (v, v2), (f, f2), (border, b2)):
        assert np.array_equal(a, b)
    with pytest.raises(ValueError, match="wings"):
        restart.decode(data[:4] + struct.pack("<i", 3) + data[8:], nx, ny, W)
    with pytest.raises(ValueError, match="bytes"):
        restart.decode(data[:-8], nx, ny, W)
    bad = bytearray(data)
    struct.pack_into("<d", bad, 8, 0.5)   # body_rel_a(1) non-zero
    with pytest.raises(ValueError, match="relative motion"):
        restart.decode(bytes(bad), nx, ny, W)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_continued_from_file_equals_continued_in_memory(gpu_lib, tmp_path, prec):
    from lbm_mutiwing_b200 import api
    from lbm_mutiwing_b200 import workloads as wl
    ep = wl.tandem_pitch_heave("r", 4.0, 2.0, 0.02, 100.0, -1.0, 0.0, 60, 40, n_wings=2, x_spacing=1.5,
                               spacing="uniform")
    with api.Simulation(ep, prec) as a, api.Simulation(ep, prec) as b:
        a.step(9, flags=api.STEP_FIELDS)
        restart.save(str(tmp_path), a, a.cycle)
        os.remove(os.path.join(str(tmp_path), restart.FILE))   # the copy is read instead
        assert restart.load(str(tmp_path), b) == a.cycle
        ra = a.step(8)
        rb = b.step(8)
        assert np.array_equal(ra, rb)
        assert np.array_equal(a.f(), b.f())
        assert np.array_equal(a.border_f0()[0], b.border_f0()[0])
