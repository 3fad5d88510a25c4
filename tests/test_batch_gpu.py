"""Packed stepping (lbm_batch_step) against stepping each episode alone.

Episodes of different lattice sizes, wing counts and step counts advance in
one batch call (long calls also time the packed bulk kernel's variants and
replay steady step pairs from CUDA graphs); every force row, the distributions, the output fields and
the running sums must equal, bit for bit, those of the same episodes
advanced one lbm_step call at a time, including over a second batch call,
a single-episode call in between, and calls that write fields or the
erranalysis velocity pair.
"""
import numpy as np
import pytest

from lbm_mutiwing_b200 import api
from lbm_mutiwing_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def small(name, wings, size, markers=60, steps=40):
    return wl.tandem_pitch_heave(name, size[0], size[1], 0.02, 100.0, -1.0, 0.0, markers, steps, n_wings=wings,
                                 x_spacing=1.5, spacing="uniform")


EPISODES = [("a", 2, (4.0, 2.0)), ("b", 1, (6.0, 3.0)), ("c", 2, (5.0, 2.0)), ("d", 3, (7.0, 2.5)),
            ("e", 1, (3.0, 2.0))]


def _pairs():
    eps = [small(*e) for e in EPISODES]
    alone = [api.Simulation(ep, api.PRECISION_FP32) for ep in eps]
    packed = [api.Simulation(ep, api.PRECISION_FP32) for ep in eps]
    return eps, alone, packed


def _same(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))


def _compare_state(sa, sb):
    _same(sa.f(), sb.f())
    ra, ca, _ = sa.sums()
    rb, cb, _ = sb.sums()
    assert ca == cb
    _same(ra, rb)


def test_batch_equals_one_at_a_time(gpu_lib):
    eps, alone, packed = _pairs()
    try:
        with api.Batch(0) as batch:
            # first call: ragged step counts, mixed flags
            ns = [5, 1, 9, 2, 6]
            fl = [0, api.STEP_FIELDS, api.STEP_ERR, api.STEP_FIELDS | api.STEP_ERR, 0]
            rows_a = [s.step(k, flags=f) for s, k, f in zip(alone, ns, fl)]
            rows_b = batch.step(packed, ns, flags=fl)
            for ra, rb in zip(rows_a, rows_b):
                _same(ra, rb)
            for k, (sa, sb) in enumerate(zip(alone, packed)):
                _compare_state(sa, sb)
                if fl[k] & api.STEP_FIELDS:
                    for xa, xb in zip(sa.output(2, 2), sb.output(2, 2)):
                        _same(xa, xb)
                if fl[k] & api.STEP_ERR and ns[k] >= 2:
                    assert sa.err() == sb.err()
            # one episode alone in between (graphs on the single path)
            _same(alone[2].step(7), packed[2].step(7))
            # second call: other counts (plane parity and geometry sets carried over)
            ns2 = [8, 3, 0, 11, 4]
            rows_a = [s.step(k) if k else None for s, k in zip(alone, ns2)]
            rows_b = batch.step(packed, ns2)
            for ra, rb, k in zip(rows_a, rows_b, ns2):
                if k:
                    _same(ra, rb)
                else:
                    assert rb is None
            for sa, sb in zip(alone, packed):
                _compare_state(sa, sb)
                assert sa.cycle == sb.cycle
            # and a subset, in another order
            sub = [3, 0]
            rows_a = [alone[i].step(6) for i in sub]
            rows_b = batch.step([packed[i] for i in sub], 6)
            for ra, rb in zip(rows_a, rows_b):
                _same(ra, rb)
            # long enough for the engine to time its bulk-kernel variants
            # (steps 1-6 each run a different one), then with the choice kept
            for _ in range(2):
                rows_a = [s.step(9) for s in alone]
                rows_b = batch.step(packed, 9)
                for ra, rb in zip(rows_a, rows_b):
                    _same(ra, rb)
            for sa, sb in zip(alone, packed):
                _compare_state(sa, sb)
    finally:
        for s in alone + packed:
            s.close()


def test_batch_rejects_bad_input(gpu_lib):
    ep = small("a", 2, (4.0, 2.0))
    with api.Simulation(ep, api.PRECISION_FP32) as s, api.Simulation(ep, api.PRECISION_FP64) as p, \
            api.Batch(0) as batch:
        with pytest.raises(api.LbmError, match="FP32"):
            batch.step([s, p], 2)
        with pytest.raises(api.LbmError, match="twice"):
            batch.step([s, s], 2)
        # the handle is untouched by the refused calls
        before = s.f()
        batch.step([s], 0)
        _same(before, s.f())


def test_substitution_forms_agree(gpu_lib):
    """The three substitutions solve the same system: the 8-row form with
    the wing's factor whole in shared memory (the default), the 8-row form
    streaming the factor through a ring of rows (wings too large for shared
    memory) and the 32-row panels built by the factorisation: on the FP64
    path, force rows within 1e-10 relative; on the FP32 path each form gives
    the same bits alone and packed."""
    ep = small("s", 2, (5.0, 2.5), markers=160)
    forms = (api.FLAG_SOLVE_STREAM, api.FLAG_SOLVE_PANELS32)
    with api.Simulation(ep, api.PRECISION_FP64) as a:
        ra = a.step(12)
    scale = np.abs(ra[:, 1:7]).max()
    for fl in forms:
        with api.Simulation(ep, api.PRECISION_FP64, flags=fl) as b:
            rb = b.step(12)
        assert np.abs(rb[:, 1:7] - ra[:, 1:7]).max() <= 1e-10 * scale, fl
    for fl in forms:
        st = api.Simulation(ep, api.PRECISION_FP32, flags=fl)
        st2 = api.Simulation(ep, api.PRECISION_FP32, flags=fl)
        try:
            rows_st = st.step(12)
            with api.Batch(0) as batch:
                _same(rows_st, batch.step([st2], 12)[0])
            _same(st.f(), st2.f())
        finally:
            st.close()
            st2.close()


def test_wing_too_large_for_shared_memory_matches_oracle(gpu_lib, oracle_lib):
    """A 500-marker wing, whose banded factor does not fit in shared memory
    whole (the substitution streams it through a ring of rows): the FP64
    path against the oracle's dense LU (1e-9 relative on forces, no-slip
    residual at solver tolerance)."""
    ep = wl.tandem_pitch_heave("big_wing", 2.4, 1.2, 0.004, 100.0, -0.4, 0.0, 500, 6, n_wings=1,
                               pitch_deg=5.0, heave=0.05, freq=2.0)
    o = oracle_lib.Oracle(ep)
    ro = o.run(1, 6)
    with api.Simulation(ep, api.PRECISION_FP64) as s:
        r64 = s.step(6)
        assert s.ibm_residual() < 1e-10
    err = np.abs(r64[:, 1:4] - ro[:, 1:4]).max() / np.abs(ro[:, 1:4]).max()
    assert err < 1e-9, err


def test_batch_graph_replay_equals_one_at_a_time(gpu_lib):
    """Long packed calls replay steady pairs of steps from CUDA graphs
    (captured on the first long stretch, reused by later calls): the same
    bits as each episode stepped alone."""
    eps = [small(n, w, size, steps=80) for n, w, size in EPISODES[:3]]
    alone = [api.Simulation(ep, api.PRECISION_FP32) for ep in eps]
    packed = [api.Simulation(ep, api.PRECISION_FP32) for ep in eps]
    try:
        with api.Batch(0) as batch:
            for _ in range(3):
                rows_a = [s.step(24) for s in alone]
                rows_b = batch.step(packed, 24)
                for ra, rb in zip(rows_a, rows_b):
                    _same(ra, rb)
            for sa, sb in zip(alone, packed):
                _compare_state(sa, sb)
    finally:
        for s in alone + packed:
            s.close()
