"""GPU parity of the WFA kernel through the C ABI: status, score and the CIGAR operation
string, bit-exact against the golden vectors (compiled WFA2-lib) and the WFA oracle."""
import json
import os

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "wfa_golden.json")


def _wfa():
    from anchorwave_b200 import wfa
    return wfa


def test_wfa_golden_single_calls(gpu):
    wfa = _wfa()
    g = json.load(open(GOLDEN))
    groups = {}
    for c in g["cases"]:
        key = (c["x"], c["o1"], c["e1"], c["o2"], c["e2"], c["singletrack"], c.get("memory_mode", 0))
        groups.setdefault(key, []).append(c)
    bad = []
    # one aligner at a time: each takes its wavefront pool from the free device memory
    for key, cases in groups.items():
        al = wfa.WfaAligner(*key[:6], memory_mode=key[6])
        for c in cases:
            st = al.align(c["target"].encode(), c["query"].encode())
            ops, score = al.cigar() if st == 0 else ("", 0)
            if (st, score, ops) != (c["result"]["status"], c["result"]["score"], c["result"]["ops"]):
                bad.append(c["name"])
        al.close()
    assert not bad, bad


@pytest.mark.parametrize("singletrack", [False, True])
@pytest.mark.parametrize("pen", [(4, 4, 2, 24, 1), (6, 8, 2, 75, 1), (2, 3, 1, 10, 1)])
def test_wfa_batch_vs_oracle(gpu, restatement, pen, singletrack):
    wfa = _wfa()
    rng = np.random.default_rng(sum(pen) + int(singletrack))
    ps, ts = [], []
    for _ in range(120):
        L = int(np.exp(rng.uniform(np.log(1), np.log(3000))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.12, 4.0)
        if rng.random() < 0.1:
            q = q.copy()
            q[rng.integers(0, len(q), 3)] = 4
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    al = wfa.WfaAligner(*pen, singletrack=singletrack)
    res, _ = al.align_batch(ps, ts)
    for p, t, r in zip(ps, ts, res):
        assert r == restatement.wfa_align(p, t, *pen, singletrack), (len(p), len(t))


def test_wfa_batched_workload_subset_vs_reference(gpu):
    """512 pairs of the 100 bp-10 kb, 0.5-5% workload against the compiled WFA2-lib."""
    wfa = _wfa()
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    ps = W.batched_wfa_set(512, seed=2)
    pats = [W.to_ascii(t) for t in ps.targets]
    txts = [W.to_ascii(q) for q in ps.queries]
    for stk in (False, True):
        al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=stk)
        res, _ = al.align_batch(pats, txts)
        for i in range(0, 512, 7):
            assert res[i] == ref.wfa_align(pats[i], txts[i], 4, 4, 2, 24, 1, singletrack=stk), i


def test_wfa_pool_retry_rounds(gpu, restatement):
    """A tiny pool forces retry rounds down to one pair at a time; results unchanged."""
    wfa = _wfa()
    rng = np.random.default_rng(99)
    ps, ts = [], []
    for _ in range(40):
        q, t = W.divergent_pair(rng, int(rng.integers(500, 2500)), 0.02, 0.05, 4.0)
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    al = wfa.WfaAligner(4, 4, 2, 24, 1, max_memory_abort=8 << 20)
    res, _ = al.align_batch(ps, ts)
    for p, t, r in zip(ps, ts, res):
        exp = restatement.wfa_align(p, t, 4, 4, 2, 24, 1, False)
        assert r == exp or r[0] == -200


def test_wfa_non_acgt_pairs(gpu, restatement):
    """Pairs with N or lowercase bases (the reference compares raw characters, so 'a' and
    'A' differ) extend byte by byte; pure uppercase ACGT pairs use the 2-bit arenas; one
    batch mixes both, and both match the oracle."""
    wfa = _wfa()
    rng = np.random.default_rng(17)
    ps, ts = [], []
    for i in range(48):
        q, t = W.divergent_pair(rng, int(rng.integers(20, 3000)), 0.0, 0.05, 4.0)
        p_, t_ = bytearray(W.to_ascii(t)), bytearray(W.to_ascii(q))
        if i % 3 == 1:
            for j in rng.integers(0, len(p_), 3):
                p_[j] = ord("N")
        elif i % 3 == 2:
            for j in rng.integers(0, len(t_), 5):
                t_[j] = t_[j] + 32  # lowercase
        ps.append(bytes(p_))
        ts.append(bytes(t_))
    al = wfa.WfaAligner(4, 4, 2, 24, 1)
    res, _ = al.align_batch(ps, ts)
    al.close()
    for p, t, r in zip(ps, ts, res):
        assert r == restatement.wfa_align(p, t, 4, 4, 2, 24, 1, False), (len(p), len(t))


def test_wfa_pool_pressure_keeps_batches(gpu):
    """Many long pairs sharing a pool too small for all of them at once: the rounds halve
    the pairs in flight instead of running them one by one, so the batch ends quickly with
    the results of a run that had the pool to spare."""
    import time
    wfa = _wfa()
    rng = np.random.default_rng(7)
    ps, ts = [], []
    for _ in range(256):
        q, t = W.divergent_pair(rng, 3000, 0.02, 0.03, 4.0)
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    big = wfa.WfaAligner(4, 4, 2, 24, 1, max_memory_abort=8 << 30)
    exp, _ = big.align_batch(ps, ts)
    big.close()
    small = wfa.WfaAligner(4, 4, 2, 24, 1, max_memory_abort=256 << 20)
    t0 = time.perf_counter()
    res, _ = small.align_batch(ps, ts)
    secs = time.perf_counter() - t0
    small.close()
    assert res == exp
    assert all(r[0] == 0 for r in res)
    assert secs < 20.0, secs


def test_align_with_wfa_mirror(gpu, restatement):
    wfa = _wfa()
    rng = np.random.default_rng(1)
    q, t = W.divergent_pair(rng, 800, 0.03, 0.03, 4.0)
    qs, ts = W.to_ascii(q).decode(), W.to_ascii(t).decode()
    st, score, aq, ar = wfa.align_with_wfa(qs, ts, -4, -4, -2, -24, -1)
    o = restatement.wfa_align(ts.encode(), qs.encode(), 4, 4, 2, 24, 1, False)
    assert st == 0 and score == o[1]
    assert aq.replace("-", "") == qs and ar.replace("-", "") == ts


@pytest.mark.parametrize("memory_mode", [1, 2])
@pytest.mark.parametrize("pen", [(4, 4, 2, 24, 1), (1, 0, 1, 0, 1), (2, 3, 1, 10, 1)])
def test_wfa_piggyback_batch_vs_oracle(gpu, restatement, pen, memory_mode):
    """Medium / low memory: ring of recent scores plus packed-CIGAR blocks on the device,
    bit-exact with the piggyback restatement (which follows the reference's offload rules;
    the device moves a cell's packed CIGAR into a block at 15 operations instead)."""
    wfa = _wfa()
    rng = np.random.default_rng(500 + sum(pen) + memory_mode)
    ps, ts = [], []
    for i in range(120):
        L = int(np.exp(rng.uniform(np.log(1), np.log(4000))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.15, 4.0)
        if i % 6 == 5:
            q, t = q % 2, t % 2  # two-letter alphabet: many equal-score paths
        if rng.random() < 0.1:
            q = q.copy()
            q[rng.integers(0, len(q), 3)] = 4
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    ps.append(b""), ts.append(b"ACGT")
    ps.append(b"ACGTA"), ts.append(b"")
    al = wfa.WfaAligner(*pen, memory_mode=memory_mode)
    res, _ = al.align_batch(ps, ts)
    al.close()
    for p, t, r in zip(ps, ts, res):
        assert r == restatement.wfa_align(p, t, *pen, memory_mode=memory_mode), (len(p), len(t))


def test_wfa_piggyback_workload_subset_vs_reference(gpu):
    """512 pairs of the 100 bp-10 kb workload in medium and low memory against the compiled
    WFA2-lib in the same modes, and against the device's high-memory results."""
    wfa = _wfa()
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    ps = W.batched_wfa_set(512, seed=3)
    pats = [W.to_ascii(t) for t in ps.targets]
    txts = [W.to_ascii(q) for q in ps.queries]
    hi = wfa.WfaAligner(4, 4, 2, 24, 1)
    exp, _ = hi.align_batch(pats, txts)
    hi.close()
    for mode in (1, 2):
        al = wfa.WfaAligner(4, 4, 2, 24, 1, memory_mode=mode)
        res, _ = al.align_batch(pats, txts)
        al.close()
        assert res == exp
        for i in range(0, 512, 11):
            assert res[i] == ref.wfa_align(pats[i], txts[i], 4, 4, 2, 24, 1, memory_mode=mode), (mode, i)


def test_wfa_piggyback_uses_less_memory(gpu):
    """Long pairs: the piggyback modes take a fraction of the high-memory mode's device
    memory per alignment (ring of the last scores plus blocks, instead of every wavefront)."""
    wfa = _wfa()
    rng = np.random.default_rng(77)
    ps, ts = [], []
    for _ in range(32):
        q, t = W.divergent_pair(rng, 8000, 0.04, 0.05, 4.0)
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    use = {}
    out = {}
    for mode in (0, 1):
        al = wfa.WfaAligner(4, 4, 2, 24, 1, memory_mode=mode)
        out[mode], _ = al.align_batch(ps, ts)
        use[mode] = al.memory()
        al.close()
    assert out[0] == out[1]
    assert all(r[0] == 0 for r in out[1])
    # 8 kb pairs at 4-5%: about 2.7x less (the ring and the blocks each take about an
    # eighth of what keeping every wavefront takes, plus allocation granularity)
    assert use[1][0] * 2 < use[0][0], use
    assert use[1][1] * 2 < use[0][1], use


def test_wfa_piggyback_pool_retry_rounds(gpu, restatement):
    """A small pool forces retry rounds in the piggyback mode too; results unchanged."""
    wfa = _wfa()
    rng = np.random.default_rng(98)
    ps, ts = [], []
    for _ in range(40):
        q, t = W.divergent_pair(rng, int(rng.integers(500, 4000)), 0.02, 0.08, 4.0)
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    al = wfa.WfaAligner(4, 4, 2, 24, 1, max_memory_abort=8 << 20, memory_mode=2)
    res, _ = al.align_batch(ps, ts)
    al.close()
    for p, t, r in zip(ps, ts, res):
        exp = restatement.wfa_align(p, t, 4, 4, 2, 24, 1, False, memory_mode=2)
        assert r == exp or r[0] == -200


def test_align_with_medium_and_low_wfa(gpu, restatement):
    wfa = _wfa()
    rng = np.random.default_rng(2)
    q, t = W.divergent_pair(rng, 1500, 0.05, 0.05, 4.0)
    qs, ts = W.to_ascii(q).decode(), W.to_ascii(t).decode()
    for fn, mode in ((wfa.align_with_medium_wfa, 1), (wfa.align_with_low_wfa, 2)):
        st, score, aq, ar = fn(qs, ts, -4, -4, -2, -24, -1)
        o = restatement.wfa_align(ts.encode(), qs.encode(), 4, 4, 2, 24, 1, False, memory_mode=mode)
        assert st == 0 and score == o[1]
        assert aq.replace("-", "") == qs and ar.replace("-", "") == ts


@pytest.mark.parametrize("singletrack", [False, True])
def test_wfa_cluster_kernel_identical(gpu, reference, singletrack):
    """Pairs whose wavefronts outgrow the width threshold leave their warp for the cluster
    kernel.  With the threshold lowered so that most pairs move, under clusters of 1, 2 and 8
    CTAs, and under the tail rule alone, every result equals the warp kernel's and the
    compiled WFA2-lib's."""
    wfa = _wfa()
    rng = np.random.default_rng(123 + int(singletrack))
    ps, ts = [], []
    for i in range(60):
        L = int(np.exp(rng.uniform(np.log(50), np.log(6000))))
        q, t = W.divergent_pair(rng, L, 0.02, 0.2, 4.0)
        if i % 5 == 0 and len(q) > 400:  # one long deletion
            at = int(rng.integers(0, len(q) - 300))
            q = np.concatenate([q[:at], q[at + int(rng.integers(50, 300)):]])
        if i % 7 == 3:
            q = q.copy()
            q[rng.integers(0, len(q), 3)] = 4
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=singletrack)
    try:
        wfa.set_wide(0)
        warp, _ = al.align_batch(ps, ts)
        assert al.launches()[1] == 0
        for width, tail, cl in ((16, 16, 1), (64, 64, 2), (256, 256, 8), (16, 16, 8), (1 << 30, 16, 8)):
            wfa.set_wide(width, tail, cl)
            got, _ = al.align_batch(ps, ts)
            n_all, n_cluster, moved = al.launches()
            # the tail rule moves only the pairs still running once few remain on warps
            assert n_cluster >= 1 and moved >= (20 if width < (1 << 30) else 1), (width, tail, cl, moved)
            assert got == warp, (width, tail, cl)
    finally:
        wfa.set_wide(8192, 1024, 8)
        al.close()
    for i in range(0, 60, 3):
        assert warp[i] == reference.wfa_align(ps[i], ts[i], 4, 4, 2, 24, 1, singletrack=singletrack), i


def test_wfa_cluster_kernel_long_pair(gpu, reference):
    """A 20 kb pair at 15% divergence (wavefronts of tens of thousands of diagonals, several
    per thread of an 8-CTA cluster) under the default threshold, standard and Singletrack,
    against the compiled WFA2-lib."""
    wfa = _wfa()
    rng = np.random.default_rng(5)
    q, t = W.divergent_pair(rng, 20000, 0.15, 0.15, 4.0)
    p_, t_ = W.to_ascii(t), W.to_ascii(q)
    for stk in (False, True):
        al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=stk)
        got, _ = al.align_batch([p_], [t_])
        assert al.launches()[2] == 1
        al.close()
        assert got[0] == reference.wfa_align(p_, t_, 4, 4, 2, 24, 1, singletrack=stk), stk


@pytest.mark.parametrize("singletrack,memory_mode", [(False, 0), (True, 0), (False, 1), (False, 2)])
def test_wfa_long_pairs_on_whole_ctas(gpu, reference, singletrack, memory_mode):
    """Long pairs run first on all four warps of a CTA (one planner thread, the diagonals over
    128 threads; in the piggyback modes every warp reserves its own block runs): with every
    pair on a CTA, with none, and with the default length threshold, the results are
    identical and equal the compiled WFA2-lib's in the same mode; in high memory a CTA's pair
    that grows too wide still moves to the cluster kernel."""
    wfa = _wfa()
    rng = np.random.default_rng(77 + int(singletrack) + 3 * memory_mode)
    ps, ts = [], []
    for i in range(48):
        L = int(np.exp(rng.uniform(np.log(20), np.log(9000))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.1, 4.0)
        if i % 6 == 0:
            q = q.copy()
            q[rng.integers(0, len(q), 2)] = 4
        ps.append(W.to_ascii(t))
        ts.append(W.to_ascii(q))
    al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=singletrack, memory_mode=memory_mode)
    try:
        wfa.set_long(0)
        wfa.set_wide(0)
        warp, _ = al.align_batch(ps, ts)
        for long_sum, width in ((1, 0), (1, 8192), (8192, 8192), (4000, 512)):
            wfa.set_long(long_sum)
            wfa.set_wide(width, min(width, 1024), 8)
            got, _ = al.align_batch(ps, ts)
            assert got == warp, (long_sum, width)
    finally:
        wfa.set_long(1536)
        wfa.set_wide(8192, 1024, 8)
        al.close()
    for i in range(0, 48, 4):
        assert warp[i] == reference.wfa_align(ps[i], ts[i], 4, 4, 2, 24, 1, singletrack=singletrack,
                                              memory_mode=memory_mode), i
