"""Re-executing a resident plan through a CUDA graph (aw_ksw_plan_execute): the first
execute runs eagerly, the second captures the launch sequence, later ones replay it.  Every
execute must give the oracle restatement's results (all ksw_extz_t fields and the CIGAR)
and still record its CUDA-event timings."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pairs(seed, n, lmin, lmax):
    """Full-width and banded pairs, so that a wave of both strip kernels is captured."""
    rng = np.random.default_rng(seed)
    qs, ts, ws = [], [], []
    for i in range(n):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        q, t = W.divergent_pair(rng, L, 0.01, 0.15, 4.0)
        qs.append(q)
        ts.append(t)
        ws.append(-1 if i % 2 else int(0.2 * max(len(q), len(t))) + 5)
    return qs, ts, ws


def _expected(restatement, qs, ts, ws, mat, zdrop=-1):
    return [restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w, zdrop=zdrop).key()
            for q, t, w in zip(qs, ts, ws)]


def test_plan_graph_replay_identical(gpu, restatement):
    qs, ts, ws = _pairs(3, 40, 100, 6000)
    mat = oracle.anchorwave_matrix(-4)
    exp = _expected(restatement, qs, ts, ws, mat)
    plan = gpu.KswPlan(qs, ts, mat, 4, 2, 24, 1, w=ws)
    plan.upload()
    used = []
    try:
        for _ in range(4):
            ms = plan.execute()
            used.append(plan.uses_graph())
            dp, _bt = plan.timing()
            assert ms > 0 and dp > 0
            assert [r.key() for r in plan.download()] == exp
    finally:
        plan.close()
    assert used == [False, True, True, True]


def test_plan_graph_recaptured_after_tuning_change(gpu, restatement):
    """A change of the warps per large pair between executes makes the plan capture again."""
    qs, ts, ws = _pairs(5, 16, 3000, 9000)
    mat = oracle.anchorwave_matrix(-4)
    exp = _expected(restatement, qs, ts, ws, mat)
    plan = gpu.KswPlan(qs, ts, mat, 4, 2, 24, 1, w=ws)
    plan.upload()
    try:
        for warps in (8, 8, 8, 4, 4, 8):
            gpu.set_tuning(warps, 4096)
            plan.execute()
            assert [r.key() for r in plan.download()] == exp, warps
        assert plan.uses_graph()
    finally:
        gpu.set_tuning(8, 4096)
        plan.close()


def test_plan_with_anti_diagonal_pairs_stays_eager(gpu, restatement):
    """z-drop pairs run on the anti-diagonal kernel, which the graph path leaves out."""
    qs, ts, ws = _pairs(7, 10, 100, 2000)
    mat = oracle.anchorwave_matrix(-4)
    exp = _expected(restatement, qs, ts, ws, mat, zdrop=200)
    plan = gpu.KswPlan(qs, ts, mat, 4, 2, 24, 1, w=ws, zdrop=200)
    plan.upload()
    try:
        for _ in range(3):
            plan.execute()
            assert not plan.uses_graph()
            assert [r.key() for r in plan.download()] == exp
    finally:
        plan.close()


def test_plan_under_deadline_stays_eager(gpu, restatement):
    qs, ts, ws = _pairs(9, 8, 100, 3000)
    mat = oracle.anchorwave_matrix(-4)
    exp = _expected(restatement, qs, ts, ws, mat)
    plan = gpu.KswPlan(qs, ts, mat, 4, 2, 24, 1, w=ws)
    plan.upload()
    try:
        plan.execute()
        plan.execute()
        assert plan.uses_graph()
        with gpu.deadline(600.0):
            plan.execute()
            assert not plan.uses_graph()
        assert [r.key() for r in plan.download()] == exp
    finally:
        plan.close()
