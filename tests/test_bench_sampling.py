"""The CPU reference's throughput estimate in bench.py (no GPU, no engine):
frame samples grow until the frame-dependent time dominates the larger one,
within the time budget, and t(n) = a + b n through them is extrapolated.
The engine is replaced by a timing model t(n) = a + b n."""
import numpy as np

import bench


def _fake(a, b, calls):
    def step(w, inp, n, seed, threads, **kw):
        calls.append(n)
        return a + b * n
    return step


def _run(monkeypatch, a, b, budget, steps=2):
    calls = []
    monkeypatch.setattr(bench, "reference_step", _fake(a, b, calls))
    w = {"n_frames": 200000}
    inp = {"quats": np.zeros((50100, 5))}
    return bench.reference_throughput(w, inp, 16, budget_s=budget, steps=steps), calls


def test_frame_part_dominates_when_the_budget_allows(monkeypatch):
    # a fixed part of 15 s and 5 ms per frame (the shape measured on a 16-core host)
    res, calls = _run(monkeypatch, 15., 0.005, budget=120.)
    assert calls[0] == 64 and max(calls) >= 4096
    assert res["frame_share"] >= 0.5
    assert abs(res["per_frame_s"] - 0.005) < 1e-9 and abs(res["fixed_s"] - 15.) < 1e-6
    assert abs(res["value"] - 50100 * 200000 / (15. + 0.005 * 200000)) < 1e-3 * res["value"]


def test_budget_bounds_the_samples(monkeypatch):
    # a slow host: the fixed part alone is 50 s; the samples stop inside the budget
    res, calls = _run(monkeypatch, 50., 0.01, budget=120.)
    assert sum(50. + 0.01 * n for n in calls) <= 120. + 1e-9 or len(calls) == 2
    assert abs(res["per_frame_s"] - 0.01) < 1e-9   # exact on a linear model


def test_repeats_only_within_the_budget(monkeypatch):
    res, calls = _run(monkeypatch, 1., 0.001, budget=30., steps=4)
    n2 = max(calls)
    assert calls.count(n2) >= 2           # the larger sample repeated
    assert sum(1. + 0.001 * n for n in calls) <= 30. + 1. + 0.001 * n2
