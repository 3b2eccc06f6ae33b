"""Autotuner for the batched and served alignment paths.

Knobs, each timed on a seeded sample of the caller's own workload (same length
distribution), the fastest installed or returned:
  * full-matrix strip kernel (aw_set_tuning): large_warps, how many warps pipeline the strips
    of one large pair (2, 4 or 8), and large_tlen_threshold, the target length from which a
    pair counts as large;
  * banded strip kernel (aw_set_band_columns): target columns per lane (4: a shorter pipeline
    lag between strips, for batches bound by their longest pair's chain; 8: less work per
    cell, for batches bound by total work; 0 keeps the per-batch rule);
  * serving loop: worker slots and the micro-batch size, chosen for the lowest p99 latency at
    a fixed offered request rate among the settings that finish the trace within 15% of the
    fastest one.  The trials should run the whole trace: a sample's tail is made of other
    requests than the trace's, and settings picked on 3,000-request samples served the whole
    trace at up to 1.6x the p99 of the best one.  The grid holds the settings that measured
    best on whole traces (one worker, four or eight workers and 256-request caps were slower).
Results are identical under every setting (tests/test_ksw2_gpu.py, tests/test_band_gpu.py and
tests/test_autotune_gpu.py check the knobs), so the choice only moves throughput and latency.
"""
from __future__ import annotations

import itertools
import threading
import time
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import ksw2

WARPS = (2, 4, 8)
THRESHOLDS = (1024, 2048, 4096, 8192)
BAND_COLUMNS = (4, 8)
SERVE_SLOTS = (2,)
SERVE_BATCH = (1024, 2048)
SERVE_SLACK = 0.15


def _sample(n: int, size: int, seed: int):
    rng = np.random.default_rng(seed)
    return rng.choice(n, size=min(size, n), replace=False) if n > size else np.arange(n)


def tune(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray], mat, q, e, q2, e2, flag: int = 0,
         sample: int = 1024, reps: int = 2, seed: int = 0) -> Tuple[Tuple[int, int], List[Dict]]:
    """Full-matrix kernel: returns ((large_warps, threshold), trials) and installs the winner."""
    idx = _sample(len(queries), sample, seed)
    qs = [queries[i] for i in idx]
    ts = [targets[i] for i in idx]
    cells = sum(len(a) * len(b) for a, b in zip(qs, ts))
    trials = []
    best = None
    for warps, thr in itertools.product(WARPS, THRESHOLDS):
        ksw2.set_tuning(warps, thr)
        plan = ksw2.KswPlan(qs, ts, mat, q, e, q2, e2, flag=flag)
        plan.upload()
        plan.execute()  # warm-up
        ms = min(plan.execute() for _ in range(reps))
        plan.close()
        trials.append({"large_warps": warps, "threshold": thr, "ms": ms, "gcups": cells / ms / 1e6})
        if best is None or ms < best[0]:
            best = (ms, warps, thr)
    ksw2.set_tuning(best[1], best[2])
    return (best[1], best[2]), trials


def tune_band(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray], bands: Sequence[int], mat, q, e, q2,
              e2, flag: int = 0, sample: int = 8, reps: int = 1, seed: int = 0,
              budget: int = 0) -> Tuple[int, List[Dict]]:
    """Banded kernel: times the sample under 4 and 8 columns per lane and under the per-batch
    rule (0); returns (columns, trials) and installs the winner.  `budget` > 0: the traceback
    budget of the trials (a share of the whole batch's, so that the sample's pairs recompute
    their tracebacks in rounds as the batch's do)."""
    idx = _sample(len(queries), sample, seed)
    qs = [queries[i] for i in idx]
    ts = [targets[i] for i in idx]
    ws = [int(bands[i]) for i in idx]
    trials = []
    best = None
    if budget > 0:
        ksw2.set_traceback_budget(budget)
    try:
        for i, cols in enumerate((0,) + BAND_COLUMNS):
            ksw2.set_band_columns(cols)
            plan = ksw2.KswPlan(qs, ts, mat, q, e, q2, e2, w=ws, flag=flag)
            plan.upload()
            if i == 0:
                plan.execute()  # warm-up: the device buffers, once for all settings
            ms = min(plan.execute() for _ in range(reps))
            plan.close()
            trials.append({"columns": cols, "ms": ms})
            if best is None or ms < best[0]:
                best = (ms, cols)
    finally:
        if budget > 0:
            ksw2.set_traceback_budget(0)
    ksw2.release_thread_buffers()
    ksw2.set_band_columns(best[1])
    return best[1], trials


def tune_serving(requests, routes, mat, q, e, q2, e2, rate: float, sample: int = 3000, hbm_budget: int = 0,
                 seed: int = 0) -> Tuple[Tuple[int, int], List[Dict]]:
    """Serving loop: every (slots, max_batch) serves a seeded sample of the routed trace with
    Poisson arrivals at `rate` requests/s; pick_serving chooses among the trials.
    Returns ((slots, max_batch), trials)."""
    from . import serve
    idx = sorted(_sample(len(requests), sample, seed).tolist())
    reqs = [requests[i] for i in idx]
    rts = [routes[i] for i in idx]
    trials = []
    for slots, batch in itertools.product(SERVE_SLOTS, SERVE_BATCH):
        rng = np.random.default_rng(seed + 1)
        with serve.AlignmentServer(mat, q, e, q2, e2, slots=slots, max_batch=batch, hbm_budget=hbm_budget) as srv:
            t0 = time.perf_counter()

            def producer():
                nxt = t0
                for k, (r, rt) in enumerate(zip(reqs, rts)):
                    nxt += rng.exponential(1.0 / rate)
                    d = nxt - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    srv.submit(k, rt.method, r.query, r.target, band=rt.band, band_max=rt.band_max,
                               window=rt.window, predicted_bytes=rt.predicted_bytes)

            th = threading.Thread(target=producer)
            th.start()
            got = 0
            while got < len(reqs):
                got += len(srv.poll(4096, wait_ms=20))
            th.join()
            dt = time.perf_counter() - t0
            st = srv.stats()
        trials.append({"slots": slots, "max_batch": batch, "requests_per_s": len(reqs) / dt,
                       "p50_ms": 1e3 * st["latency_p50_s"], "p99_ms": 1e3 * st["latency_p99_s"],
                       "seconds": dt})
    ksw2.release_thread_buffers()
    return pick_serving(trials), trials


def pick_serving(trials: List[Dict], slack: float = SERVE_SLACK) -> Tuple[int, int]:
    """The (slots, max_batch) of the trial with the lowest p99 latency among those whose sample
    finished within `slack` of the fastest trial."""
    fastest = min(t["seconds"] for t in trials)
    keep = [t for t in trials if t["seconds"] <= (1.0 + slack) * fastest]
    best = min(keep, key=lambda t: (t["p99_ms"], t["seconds"]))
    return best["slots"], best["max_batch"]
