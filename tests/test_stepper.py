"""Continuous batching logic of batch.PackedStepper on the CPU, with a fake
packed engine: segments longer than a round are split, requests arriving
while a round runs join the next one, the last round carries the caller's
flags, rows come back in order, and a failing episode fails alone."""
import threading
import time

import numpy as np
import pytest

from lbm_mutiwing_b200 import api
from lbm_mutiwing_b200.batch import PackedStepper


class FakeSim:
    def __init__(self, name, row_len=4):
        self.name, self.row_len, self.cycle = name, row_len, 1
        self.calls = []          # (first_cycle, n, flags) per round
        self.fail_at = None

    def step(self, n, first_cycle=None, rows=True, flags=0):   # the one-episode round
        time.sleep(0.02)
        return FakeBatch.rows_for(self, n, first_cycle, flags)


class FakeBatch:
    def __init__(self, delay=0.02):
        self.delay, self.rounds, self.closed = delay, [], False

    @staticmethod
    def rows_for(sim, n, first, flags):
        if sim.fail_at is not None and first <= sim.fail_at < first + n:
            raise api.LbmError(f"{sim.name} failed")
        sim.calls.append((first, n, flags))
        sim.cycle = first + n
        # row r carries the cycle it stands for
        return np.repeat((first + np.arange(n, dtype=float))[:, None], sim.row_len, axis=1)

    def step(self, sims, n_steps, first_cycles=None, rows=True, flags=0):
        self.rounds.append([s.name for s in sims])
        time.sleep(self.delay)
        outs, rcs, msgs = [], [], []
        for s, k, f0, fl in zip(sims, n_steps, first_cycles, flags):
            try:
                outs.append(self.rows_for(s, k, f0, fl))
                rcs.append(0)
                msgs.append("")
            except api.LbmError as e:
                outs.append(None)
                rcs.append(1)
                msgs.append(str(e))
        if any(rcs):
            raise api.BatchStepError("episode failed", rcs, msgs, outs)
        return outs

    def close(self):
        self.closed = True


def test_rounds_split_and_join():
    fb = FakeBatch()
    st = PackedStepper(chunk=10, batch=fb)
    a, b = FakeSim("a"), FakeSim("b")
    out = {}
    try:
        ta = threading.Thread(target=lambda: out.__setitem__("a", st.step(a, 35, first_cycle=1, flags=3)))
        ta.start()
        time.sleep(0.03)           # b arrives while a's first round runs
        out["b"] = st.step(b, 12, first_cycle=5, flags=1)
        ta.join()
    finally:
        st.close()
    assert fb.closed
    # a: 35 steps in rounds of 10 with the flags on the last round only
    assert a.calls == [(1, 10, 0), (11, 10, 0), (21, 10, 0), (31, 5, 3)]
    assert [c[1] for c in b.calls] == [10, 2] and b.calls[-1][2] == 1 and b.calls[0][0] == 5
    # rows in order, one per cycle
    assert np.array_equal(out["a"][:, 0], np.arange(1, 36)) and np.array_equal(out["b"][:, 0], np.arange(5, 17))
    assert a.cycle == 36 and b.cycle == 17
    # b joined a running batch: some round packs both episodes
    assert any(sorted(r) == ["a", "b"] for r in fb.rounds)


def test_failing_episode_fails_alone():
    fb = FakeBatch(delay=0.0)
    st = PackedStepper(chunk=8, batch=fb)
    a, b = FakeSim("a"), FakeSim("b")
    b.fail_at = 12
    res = {}

    def run(name, sim):
        try:
            res[name] = st.step(sim, 20, first_cycle=1)
        except api.LbmError as e:
            res[name] = e
    try:
        ts = [threading.Thread(target=run, args=(n, s)) for n, s in (("a", a), ("b", b))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    finally:
        st.close()
    assert isinstance(res["b"], api.LbmError) and "b failed" in str(res["b"])
    # a keeps every row, including those of the round in which b failed
    assert np.array_equal(res["a"][:, 0], np.arange(1, 21))


def test_zero_steps_go_straight_to_the_episode():
    st = PackedStepper(chunk=8, batch=FakeBatch())
    try:
        a = FakeSim("a")
        assert st.step(a, 0, first_cycle=3).shape == (0, 4)
    finally:
        st.close()
