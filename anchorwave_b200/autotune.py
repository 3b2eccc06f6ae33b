"""Autotuner for the batched KSW2 path.

Two launch knobs decide how a batch maps onto the SMs (aw_set_tuning):
  * large_warps: how many warps pipeline the strips of one large pair (1, 2, 4 or 8);
  * large_tlen_threshold: the target length from which a pair counts as large.
The tuner times a seeded sample of the caller's workload (same length distribution) under
every candidate with CUDA events on the plan's stream, keeps the fastest, and installs it.
Results are identical under every setting (tests/test_ksw2_gpu.py checks the knobs), so
the choice only moves throughput.
"""
from __future__ import annotations

import itertools
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import ksw2

WARPS = (2, 4, 8)
THRESHOLDS = (1024, 2048, 4096, 8192)


def tune(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray], mat, q, e, q2, e2, flag: int = 0,
         sample: int = 1024, reps: int = 2, seed: int = 0) -> Tuple[Tuple[int, int], List[Dict]]:
    """Returns ((large_warps, threshold), trials) and installs the winner."""
    n = len(queries)
    rng = np.random.default_rng(seed)
    idx = rng.choice(n, size=min(sample, n), replace=False) if n > sample else np.arange(n)
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
