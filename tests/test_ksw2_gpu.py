"""GPU parity of the KSW2 kernels through the C ABI (libaw_b200.so), bit-exact against the
golden vectors (compiled reference) and against the oracle on seeded corpora: every
ksw_extz_t field and the CIGAR words, including tie-breaking."""
import json
import os
import threading

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ksw2_golden.json")
FIELDS = ("max", "zdropped", "max_q", "max_t", "mqe", "mqe_t", "mte", "mte_q", "score", "n_cigar", "reach_end",
          "stopped", "cigar")


def _codes(s):
    return W.to_codes(s.encode())


def _mat(c):
    return c.get("mat") or oracle.anchorwave_matrix(c["mismatch"])


def _as_dict(r):
    return {k: getattr(r, k) for k in FIELDS}


def test_golden_single_calls(gpu):
    g = json.load(open(GOLDEN))
    bad = []
    for c in g["cases"]:
        fn = gpu.ksw_extd2_singletrack if c["variant"] == 2 else gpu.ksw_extd2
        r = fn(_codes(c["query"]), _codes(c["target"]), _mat(c), c["q"], c["e"], c["q2"], c["e2"], w=c["w"],
               zdrop=c["zdrop"], end_bonus=c["end_bonus"], flag=c["flag"])
        if _as_dict(r) != c["result"]:
            bad.append(c["name"])
    assert not bad, f"GPU differs from golden on {bad}"


def test_golden_batched(gpu):
    """The same golden cases through one batched submission per parameter group."""
    g = json.load(open(GOLDEN))
    groups = {}
    for c in g["cases"]:
        if c["variant"] == 2:
            continue
        key = (tuple(_mat(c)), c["q"], c["e"], c["q2"], c["e2"], c["zdrop"], c["end_bonus"], c["flag"])
        groups.setdefault(key, []).append(c)
    for key, cs in groups.items():
        mat, q, e, q2, e2, zdrop, eb, flag = key
        res = gpu.ksw_extd2_batch([_codes(c["query"]) for c in cs], [_codes(c["target"]) for c in cs], list(mat), q,
                                  e, q2, e2, w=[c["w"] for c in cs], zdrop=zdrop, end_bonus=eb, flag=flag)
        for c, r in zip(cs, res):
            assert _as_dict(r) == c["result"], c["name"]


PEN = [(4, 2, 24, 1), (8, 2, 75, 1), (6, 1, 20, 0), (2, 3, 30, 1)]


def _random_set(seed, n, lmin, lmax, band=False, nfrac=0.0):
    rng = np.random.default_rng(seed)
    qs, ts, ws = [], [], []
    for _ in range(n):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        q, t = W.divergent_pair(rng, L, 0.01, 0.25, 4.0)
        if nfrac and rng.random() < nfrac:
            q = q.copy()
            q[rng.integers(0, len(q), 4)] = 4
        qs.append(q)
        ts.append(t)
        ws.append(int(rng.integers(0, max(2, L // 4))) if band else -1)
    return qs, ts, ws


@pytest.mark.parametrize("pen", PEN)
@pytest.mark.parametrize("flag", [0, 0x01, 0x02, 0x80, 0x800])
def test_full_random_vs_restatement(gpu, restatement, pen, flag):
    qs, ts, ws = _random_set(100 + flag + pen[0], 60, 1, 1200)
    res = gpu.ksw_extd2_batch(qs, ts, oracle.anchorwave_matrix(-4), *pen, flag=flag)
    for q, t, r in zip(qs, ts, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), *pen, flag=flag)
        assert r.key() == o.key(), (len(q), len(t), pen, hex(flag))


def test_generic_scoring_with_n(gpu, restatement):
    qs, ts, _ = _random_set(7, 80, 20, 900, nfrac=0.5)
    res = gpu.ksw_extd2_batch(qs, ts, oracle.anchorwave_matrix(-4), 4, 2, 24, 1, flag=oracle.KSW_EZ_GENERIC_SC)
    for q, t, r in zip(qs, ts, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1,
                                  flag=oracle.KSW_EZ_GENERIC_SC)
        assert r.key() == o.key()


@pytest.mark.parametrize("flag", [0, 0x01, 0x02, 0x1000, 0x40, 0x08])
def test_banded_random_vs_restatement(gpu, restatement, flag):
    qs, ts, ws = _random_set(31 + flag, 40, 10, 900, band=True)
    for q, t, w in zip(qs, ts, ws):
        fn = gpu.ksw_extd2_singletrack if flag & 0x1000 else gpu.ksw_extd2
        r = fn(q, t, oracle.anchorwave_matrix(-4), 4, 2, 24, 1, w=w, flag=flag & ~0x1000)
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1, w=w,
                                  flag=flag)
        assert r.key() == o.key(), (len(q), len(t), w, hex(flag))


def test_batched_full_subset_vs_reference(gpu):
    """512 pairs of the batched 200 bp-20 kb workload, all fields + CIGAR via the per-pair hash."""
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    ps = W.batched_full_set(512, seed=1)
    mat = oracle.anchorwave_matrix(-4)
    res = gpu.ksw_extd2_batch(ps.queries, ps.targets, mat, 4, 2, 24, 1)
    cpu = ref.ksw_batch([q.tobytes() for q in ps.queries], [t.tobytes() for t in ps.targets], mat, 4, 2, 24, 1)
    hashes = [oracle.result_hash(r) for r in res]
    bad = [i for i, h in enumerate(hashes) if h != int(cpu["hash"][i])]
    assert not bad, f"{len(bad)} pairs differ, first {bad[:5]}"


@pytest.mark.parametrize("warps", [1, 2, 4, 8])
def test_multiwarp_pipeline_and_waves(gpu, restatement, warps):
    """Strip pipelining across W warps and the traceback-wave split give identical results."""
    qs, ts, _ = _random_set(55, 24, 300, 4000)
    mat = oracle.anchorwave_matrix(-4)
    try:
        gpu.set_tuning(large_warps=warps, large_tlen_threshold=256)
        gpu.set_traceback_budget(64 << 20)  # forces several waves
        res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1)
    finally:
        gpu.set_tuning(large_warps=8, large_tlen_threshold=4096)
        gpu.set_traceback_budget(0)
    for q, t, r in zip(qs, ts, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1)
        assert r.key() == o.key()


def test_repeated_batches_with_many_waves(gpu, restatement):
    """Back-to-back batch calls on one thread whose plans need more and more traceback waves
    (every wave has its own work-queue counters, all reset per call)."""
    qs, ts, _ = _random_set(123, 40, 300, 3000)
    mat = oracle.anchorwave_matrix(-4)
    exp = [restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1).key() for q, t in zip(qs, ts)]
    try:
        for budget in (256 << 20, 64 << 20, 24 << 20, 12 << 20, 64 << 20):
            gpu.set_traceback_budget(budget)
            res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1)
            assert [r.key() for r in res] == exp, budget
    finally:
        gpu.set_traceback_budget(0)


def test_plan_repeatable(gpu):
    ps = W.batched_full_set(64, seed=9, lmax=3000)
    plan = gpu.KswPlan(ps.queries, ps.targets, oracle.anchorwave_matrix(-4), 4, 2, 24, 1)
    plan.upload()
    plan.execute()
    a = [r.key() for r in plan.download()]
    plan.execute()
    b = [r.key() for r in plan.download()]
    plan.close()
    assert a == b


def test_threads_are_independent(gpu):
    """Concurrent host threads each get their own stream/buffers; results equal serial calls."""
    qs, ts, _ = _random_set(77, 16, 100, 2000)
    mat = oracle.anchorwave_matrix(-4)
    serial = [gpu.ksw_extd2(q, t, mat, 4, 2, 24, 1).key() for q, t in zip(qs, ts)]
    out = [None] * len(qs)

    def worker(k):
        for i in range(k, len(qs), 4):
            out[i] = gpu.ksw_extd2(qs[i], ts[i], mat, 4, 2, 24, 1).key()

    th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert out == serial


def test_anchorwave_wrappers(gpu, restatement):
    rng = np.random.default_rng(4)
    q, t = W.divergent_pair(rng, 600, 0.05, 0.05, 3.0)
    qs, ts = W.to_ascii(q).decode(), W.to_ascii(t).decode()
    score, aq, ad = gpu.minimap2_alignment(qs, ts, 0, -4, -4, -2, -24, -1)
    o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1)
    assert score == o.score and aq.replace("-", "") == qs and ad.replace("-", "") == ts
    s2, _ = gpu.ksw2_score_only(qs, ts, -4, -4, -2, -24, -1)
    assert s2 == o.score
    s3, aq3, ad3, stopped = gpu.align_ksw2_singletrack(qs, ts, -4, -4, -2, -24, -1)
    assert not stopped and s3 == o.score


def test_exact_kernel_generic_scores(gpu, restatement):
    """Z-drop sends pairs to the exact anti-diagonal kernel; with KSW_EZ_GENERIC_SC its score
    fill reads the matrix with the reversed-query index (regression: it read the forward
    query there), with and without the Singletrack traceback, left and right aligned."""
    rng = np.random.default_rng(404)
    mat = [2 if a == b else (-4 if a < 4 and b < 4 else -1) for a in range(5) for b in range(5)]
    for i in range(60):
        L = int(np.exp(rng.uniform(np.log(2), np.log(1500))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.2, 4.0)
        flag = oracle.KSW_EZ_GENERIC_SC | (oracle.KSW_EZ_RIGHT if i % 2 else 0)
        w = -1 if i % 3 else int(rng.integers(1, max(2, L // 2)))
        for st in (False, True):
            f = gpu.ksw_extd2_singletrack if st else gpu.ksw_extd2
            g = f(q, t, mat, 4, 2, 24, 1, w=w, zdrop=200, flag=flag)
            o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w, zdrop=200,
                                      flag=flag | (oracle.KSW_EZ_SINGLETRACK if st else 0), block=64)
            assert g.key() == o.key(), (i, L, w, hex(flag), st)


@pytest.mark.parametrize("flag", [0, 0x02, 0x01, 0x800])
def test_long_full_pair_on_the_banded_kernel(gpu, restatement, flag):
    """A long full-matrix pair alone (the batch's critical path) runs on the banded kernel at
    full width; with the routing off it runs on the strip kernel.  Both give the oracle's
    ksw_extz_t and CIGAR."""
    rng = np.random.default_rng(60 + flag)
    q, t = W.divergent_pair(rng, 24000, 0.03, 0.06, 4.0)
    mat = oracle.anchorwave_matrix(-4)
    exp = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, flag=flag).key()
    try:
        for on in (True, False):
            gpu.set_full_pair_routing(on)
            assert gpu.ksw_extd2(q, t, mat, 4, 2, 24, 1, flag=flag).key() == exp, on
            assert gpu.ksw_extd2_batch([q], [t], mat, 4, 2, 24, 1, flag=flag)[0].key() == exp, on
    finally:
        gpu.set_full_pair_routing(True)
