"""Two-step passes of the fused path against single steps.

A pass advances the lattice n -> n + 2 with one read of step n's planes
(temporal blocking); the band nodes and the border of step n + 1 come from
the first step's immersed boundary and far field, every other node of step
n + 1 is recomputed where it is needed.  Each node is computed by the same
collision code, so stepping in passes must give, bit for bit, the force
rows, distributions, running sums and output fields of stepping one step at
a time (LBM_FLAG_SINGLE_STEPS), and the no-slip residual of each call's last
step (a call without field requests ends in a pass, which computes it), for
odd and even step counts, calls that continue one another, eager launches
and CUDA graph replay, wings close to tile edges, coupled wings and a
lattice made only of border tiles; with both tile shapes a handle may take
(64 x 8, and 64 x 12 as on large lattices).
"""
import numpy as np
import pytest

from lbm_mutiwing_b200 import api
from lbm_mutiwing_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def small(name, wings, size, markers=60, steps=80, x_spacing=1.5):
    return wl.tandem_pitch_heave(name, size[0], size[1], 0.02, 100.0, -1.0, 0.0, markers, steps, n_wings=wings,
                                 x_spacing=x_spacing, spacing="uniform")


def _same(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))


def _run(ep, calls, flags=0, graphs=True, step_flags=0):
    with api.Simulation(ep, api.PRECISION_FP32, flags=flags, graphs=graphs) as s:
        rows = []
        cyc = 1
        for n in calls:
            rows.append(s.step(n, first_cycle=cyc, flags=step_flags))
            cyc += n
        out = {"rows": np.concatenate(rows), "f": s.f(), "sums": s.sums(), "resid": s.ibm_residual()}
        if step_flags & api.STEP_FIELDS:
            out["fields"] = s.fields()
    return out


def _compare(a, b):
    _same(a["rows"], b["rows"])
    _same(a["f"], b["f"])
    ra, ca, _ = a["sums"]
    rb, cb, _ = b["sums"]
    assert ca == cb
    _same(ra, rb)
    assert a["resid"] == b["resid"]   # the no-slip residual of the call's last step
    for x, y in zip(a.get("fields", ()), b.get("fields", ())):
        _same(x, y)


@pytest.mark.parametrize("calls", [[1], [2], [3], [4], [5], [9], [26], [7, 8, 1, 12]])
def test_passes_equal_single_steps(gpu_lib, calls):
    ep = small("p", 2, (5.0, 2.5))
    _compare(_run(ep, calls), _run(ep, calls, flags=api.FLAG_SINGLE_STEPS))


@pytest.mark.parametrize("graphs", [True, False])
def test_passes_equal_single_steps_eager_and_fields(gpu_lib, graphs):
    ep = small("q", 3, (7.0, 2.5))
    _compare(_run(ep, [11, 10], graphs=graphs, step_flags=api.STEP_FIELDS),
             _run(ep, [11, 10], flags=api.FLAG_SINGLE_STEPS, step_flags=api.STEP_FIELDS))


def test_passes_with_wings_across_tile_edges(gpu_lib):
    """Two wings at 1.28 chords with 64-node chords: their bands straddle
    pass tile columns and rows over the run."""
    ep = wl.tandem_pitch_heave("edges", 6.0, 3.0, 1.0 / 64.0, 100.0, -1.5, 0.0, 120, 40, n_wings=2,
                               x_spacing=1.28, spacing="uniform", pitch_deg=20.0, heave=0.3, freq=2.0)
    _compare(_run(ep, [40]), _run(ep, [40], flags=api.FLAG_SINGLE_STEPS))


def test_passes_coupled_wings(gpu_lib):
    """Wings whose supports share nodes: the joint solve runs in both chains
    of every pass."""
    ep = wl.tandem_pitch_heave("coupled", 5.0, 2.5, 0.02, 100.0, -1.0, 0.0, 100, 20, n_wings=2,
                               x_spacing=1.03, lag=0.0, pitch_deg=3.0, heave=0.1, freq=1.0)
    _compare(_run(ep, [20]), _run(ep, [20], flags=api.FLAG_SINGLE_STEPS))


def test_passes_small_lattice_all_border_tiles(gpu_lib):
    """A 27 x 19 lattice with one 10-node wing: every tile's ring meets the
    border, so every tile is a near tile."""
    ep = wl.tandem_pitch_heave("tiny", 2.6, 1.8, 0.1, 100.0, -0.4, 0.0, 30, 12, n_wings=1, pitch_deg=2.0,
                               heave=0.02)
    assert (ep.nx, ep.ny) == (27, 19)
    _compare(_run(ep, [12]), _run(ep, [12], flags=api.FLAG_SINGLE_STEPS))


TALL = api.FLAG_PASS_TALL_TILES


@pytest.mark.parametrize("calls", [[2], [5], [26], [7, 8, 1, 12]])
def test_tall_tiles_equal_single_steps(gpu_lib, calls):
    ep = small("pt", 2, (5.0, 2.5))
    _compare(_run(ep, calls, flags=TALL), _run(ep, calls, flags=api.FLAG_SINGLE_STEPS))


def test_tall_tiles_fields_and_eager(gpu_lib):
    ep = small("qt", 3, (7.0, 2.5))
    _compare(_run(ep, [11, 10], flags=TALL | api.FLAG_NO_GRAPHS, step_flags=api.STEP_FIELDS),
             _run(ep, [11, 10], flags=api.FLAG_SINGLE_STEPS, step_flags=api.STEP_FIELDS))


def test_tall_tiles_wings_across_tile_edges(gpu_lib):
    ep = wl.tandem_pitch_heave("edges_t", 6.0, 3.0, 1.0 / 64.0, 100.0, -1.5, 0.0, 120, 40, n_wings=2,
                               x_spacing=1.28, spacing="uniform", pitch_deg=20.0, heave=0.3, freq=2.0)
    _compare(_run(ep, [40], flags=TALL), _run(ep, [40], flags=api.FLAG_SINGLE_STEPS))


def test_tall_tiles_coupled_wings_and_small_lattice(gpu_lib):
    ep = wl.tandem_pitch_heave("coupled_t", 5.0, 2.5, 0.02, 100.0, -1.0, 0.0, 100, 20, n_wings=2,
                               x_spacing=1.03, lag=0.0, pitch_deg=3.0, heave=0.1, freq=1.0)
    _compare(_run(ep, [20], flags=TALL), _run(ep, [20], flags=api.FLAG_SINGLE_STEPS))
    ep = wl.tandem_pitch_heave("tiny_t", 2.6, 1.8, 0.1, 100.0, -0.4, 0.0, 30, 12, n_wings=1, pitch_deg=2.0,
                               heave=0.02)
    _compare(_run(ep, [12], flags=TALL), _run(ep, [12], flags=api.FLAG_SINGLE_STEPS))
