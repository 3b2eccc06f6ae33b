"""GPU tests of the autotuner: the settings it installs for the full-matrix and the banded
strip kernels leave every result bit-exact with the oracle, and the serving tuner returns a
setting from its grid with its trials."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import autotune, ksw2
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
PEN = (4, 2, 24, 1)


def test_tuned_full_kernel_results_identical(gpu, restatement):
    ps = W.batched_full_set(48, seed=31, lmin=200, lmax=6000)
    mat = oracle.anchorwave_matrix(-4)
    try:
        (warps, thr), trials = autotune.tune(ps.queries, ps.targets, mat, *PEN, sample=48, reps=1)
        assert len(trials) == len(autotune.WARPS) * len(autotune.THRESHOLDS)
        res = gpu.ksw_extd2_batch(ps.queries, ps.targets, mat, *PEN)
    finally:
        gpu.set_tuning(8, 4096)
    for q, t, r in zip(ps.queries, ps.targets, res):
        assert r.key() == restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *PEN).key()


def test_tuned_band_columns_results_identical(gpu, restatement):
    rng = np.random.default_rng(5)
    qs, ts, ws = [], [], []
    for _ in range(6):
        q, t = W.divergent_pair(rng, int(rng.integers(3000, 9000)), 0.02, 0.1, 4.0)
        qs.append(q), ts.append(t), ws.append(int(0.1 * min(len(q), len(t))))
    mat = oracle.anchorwave_matrix(-4)
    try:
        cols, trials = autotune.tune_band(qs, ts, ws, mat, *PEN, sample=6)
        assert cols in (0, 4, 8) and len(trials) == 3
        res = gpu.ksw_extd2_batch(qs, ts, mat, *PEN, w=ws)
    finally:
        gpu.set_band_columns(0)
    for q, t, w, r in zip(qs, ts, ws, res):
        assert r.key() == restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *PEN, w=w).key()


def test_serving_tuner_returns_a_grid_setting(gpu):
    from anchorwave_b200 import serve
    reqs = W.serving_trace(120, seed=8, lmax=5000)
    routes = [serve.ServeRouteSpec(0, -1) for _ in reqs]
    (slots, batch), trials = autotune.tune_serving(reqs, routes, ksw2.anchorwave_matrix(-4), *PEN, rate=400.0,
                                                   sample=120, hbm_budget=8 << 30)
    assert slots in autotune.SERVE_SLOTS and batch in autotune.SERVE_BATCH
    assert len(trials) == len(autotune.SERVE_SLOTS) * len(autotune.SERVE_BATCH)
    assert all(t["p99_ms"] >= t["p50_ms"] > 0 for t in trials)
