"""Host logic of the multi-problem batch: the longest-first assignment, the
plan chosen from measured times, and the autotuner's cache (no GPU: the
measurements are a fixed table)."""
import json

import numpy as np


def test_lpt_assignment_and_makespan():
    from waveforminversionust_b200.batch import lpt
    groups, span = lpt([5.0, 3.0, 3.0, 2.0, 2.0, 1.0], 2)
    assert sorted(sum(groups, [])) == list(range(6))
    loads = [sum([5.0, 3.0, 3.0, 2.0, 2.0, 1.0][i] for i in g) for g in groups]
    assert span == max(loads) == 8.0
    assert groups == lpt([5.0, 3.0, 3.0, 2.0, 2.0, 1.0], 2)[0]          # deterministic
    assert lpt([], 3) == ([[], [], []], 0.0)


def test_plan_shares_small_problems_and_keeps_large_ones_alone():
    from waveforminversionust_b200.batch import plan
    # two large problems gain nothing from a partition (or do not fit one),
    # six small ones run at nearly the same speed on a quarter of the GPU
    t_full = [0.09, 0.08, 0.02, 0.02, 0.018, 0.018, 0.016, 0.016]
    t_part = {2: [0.2, 0.19, 0.022, 0.022, 0.02, 0.02, 0.018, 0.018],
              4: [None, None, 0.025, 0.025, 0.023, 0.023, 0.02, 0.02]}
    pl = plan(t_full, t_part, 148)
    assert pl.parts == 4 and pl.cap == 37
    assert pl.exclusive == [0, 1]
    assert sorted(i for g in pl.groups for i in g) == [2, 3, 4, 5, 6, 7]
    assert abs(pl.predicted_s - (0.17 + 0.043)) < 1e-12
    assert pl.predicted_s < sum(t_full)
    # nothing to gain: everything alone, in order
    slow = {2: [2 * t for t in t_full], 4: [4 * t for t in t_full]}
    pl1 = plan(t_full, slow, 148)
    assert pl1.parts == 1 and pl1.exclusive == list(range(8))


def test_autotuner_is_deterministic_and_caches(tmp_path, monkeypatch):
    from waveforminversionust_b200 import batch
    from waveforminversionust_b200.batch import Autotuner, BatchProblem

    def prob(n, n_tx, f):
        x = np.arange(n) * 3e-4
        return BatchProblem(x, x, np.full((n, n), 1500.0), f, 16 * 3e-4, np.arange(1, n_tx + 1),
                            np.arange(1, n_tx + 1), np.zeros((n_tx, n_tx), complex), np.ones((n_tx, n_tx), bool))
    problems = [prob(552, 256, 1.2e6), prob(160, 16, 0.5e6), prob(160, 32, 0.6e6), prob(224, 64, 0.8e6)]
    calls = []

    def fake(self, p, cap, chunks=0):
        key = self._key(p, cap, chunks)
        if key in self.cache:
            return self.cache[key]
        calls.append(key)
        ny = p.shape[0]
        if cap and ny > 400 and cap < 135:
            t = None                                  # the large grid does not fit a partition
        else:
            base = 1e-7 * ny * ny * (1 + p.tx_index.size / 64)
            t = base * (1.0 if not cap else 1.0 + 0.1 * (148 // cap)) * (0.9 if chunks == 12 else 1.0)
        self.cache[key] = t
        return t
    monkeypatch.setattr(Autotuner, "measure", fake)
    path = tmp_path / "tune.json"
    a = Autotuner(cache_path=str(path))
    pl = a.tune(problems, n_sm=148)
    n_calls = len(calls)
    assert 0 in pl.exclusive and pl.parts > 1
    assert json.loads(path.read_text())
    b = Autotuner(cache_path=str(path))              # a second tuner answers from the file
    pl2 = b.tune(problems, n_sm=148)
    assert len(calls) == n_calls
    assert (pl2.parts, pl2.exclusive, pl2.groups, pl2.chunks) == (pl.parts, pl.exclusive, pl.groups, pl.chunks)
