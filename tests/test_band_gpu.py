"""GPU parity of the banded strip kernel (banded ksw_extd2 and the Singletrack traceback)
through the C ABI, bit-exact against the oracle restatement (the reference's padding-lane
semantics at the AVX-512 block of 64) and against the compiled reference: every ksw_extz_t
field and the CIGAR words."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

PEN = [(4, 2, 24, 1), (8, 2, 75, 1), (6, 1, 20, 0), (2, 3, 30, 1), (24, 1, 4, 2)]
SCORE_ONLY, RIGHT, GENERIC, REV, SEMI, ST = 0x01, 0x02, 0x04, 0x80, 0x800, 0x1000


def _pairs(seed, n, lmin, lmax, wfrac=(0.0, 0.5), nfrac=0.0, dmax=0.25):
    rng = np.random.default_rng(seed)
    qs, ts, ws = [], [], []
    for _ in range(n):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        q, t = W.divergent_pair(rng, max(L, 1), 0.01, dmax, 4.0)
        if rng.random() < 0.3 and len(q) > 60:
            at = int(rng.integers(0, len(q) - 50))
            q = np.concatenate([q[:at], q[at + int(rng.integers(1, 50)):]])
        if nfrac and rng.random() < nfrac:
            q = q.copy()
            q[rng.integers(0, len(q), 3)] = 4
            t = t.copy()
            t[rng.integers(0, len(t), 3)] = 4
        qs.append(q)
        ts.append(t)
        ws.append(int(rng.uniform(*wfrac) * max(len(q), len(t))) + int(rng.integers(0, 20)))
    return qs, ts, ws


def _check(gpu, restatement, qs, ts, ws, pen, flag, mat=None):
    mat = mat or oracle.anchorwave_matrix(-4)
    res = gpu.ksw_extd2_batch(qs, ts, mat, *pen, w=ws, flag=flag)
    bad = []
    for k, (q, t, w, r) in enumerate(zip(qs, ts, ws, res)):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w, flag=flag)
        if r.key() != o.key():
            bad.append((k, len(q), len(t), w))
    assert not bad, f"{len(bad)} of {len(qs)} differ, first {bad[:4]} flag={hex(flag)} pen={pen}"


@pytest.fixture(params=[8, 4], ids=["cols8", "cols4"])
def columns(request, gpu):
    gpu.set_band_columns(request.param)
    yield request.param
    gpu.set_band_columns(0)


@pytest.mark.parametrize("pen", PEN)
@pytest.mark.parametrize("flag", [0, SCORE_ONLY, RIGHT, REV, SEMI])
def test_banded_batch_vs_restatement(gpu, restatement, columns, pen, flag):
    qs, ts, ws = _pairs(1000 + flag + pen[0], 48, 1, 1500)
    _check(gpu, restatement, qs, ts, ws, pen, flag)


@pytest.mark.parametrize("flag", [0, RIGHT])
def test_banded_generic_scoring_with_n(gpu, restatement, columns, flag):
    qs, ts, ws = _pairs(77 + flag, 40, 10, 1200, nfrac=0.6)
    _check(gpu, restatement, qs, ts, ws, (4, 2, 24, 1), GENERIC | flag)


@pytest.mark.parametrize("pen", PEN[:3])
@pytest.mark.parametrize("banded", [False, True])
def test_singletrack_vs_restatement(gpu, restatement, columns, pen, banded):
    qs, ts, ws = _pairs(300 + pen[0] + banded, 40, 1, 1500, wfrac=(0.02, 0.6) if banded else (1.0, 1.0))
    _check(gpu, restatement, qs, ts, ws if banded else [-1] * len(qs), pen, ST)


def test_singletrack_single_calls(gpu, restatement):
    qs, ts, ws = _pairs(5, 12, 50, 3000, wfrac=(0.05, 0.3))
    mat = oracle.anchorwave_matrix(-4)
    for q, t, w in zip(qs, ts, ws):
        r = gpu.ksw_extd2_singletrack(q, t, mat, 4, 2, 24, 1, w=w)
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w, flag=ST)
        assert r.key() == o.key(), (len(q), len(t), w)


def test_band_break_and_tiny(gpu, restatement, columns):
    """Bands too narrow to reach the end (zdropped, KSW_NEG_INF score), w = 0..3 and
    one-base sequences."""
    rng = np.random.default_rng(11)
    qs, ts, ws = [], [], []
    for _ in range(60):
        tl = int(rng.integers(1, 400))
        ql = max(1, tl + int(rng.integers(-300, 300)))
        qs.append(rng.integers(0, 4, ql).astype(np.uint8))
        ts.append(rng.integers(0, 4, tl).astype(np.uint8))
        ws.append(int(rng.integers(0, 4)) if rng.random() < 0.3 else int(rng.integers(0, 200)))
    for flag in (0, SCORE_ONLY, ST):
        _check(gpu, restatement, qs, ts, ws, (4, 2, 24, 1), flag)


def test_long_banded_vs_restatement(gpu, restatement, columns):
    """Multi-strip pairs whose strips run on many warps at once, with long indels."""
    rng = np.random.default_rng(21)
    qs, ts, ws = [], [], []
    for L in (6000, 9000, 14000):
        t = W.random_dna(rng, L)
        q = W.repeat_query(rng, t, long_indels=(1, 3), long_max=L // 20, element=L // 10)
        qs.append(q)
        ts.append(t)
        ws.append(int(0.1 * min(len(q), len(t))))
    for flag in (0, ST):
        _check(gpu, restatement, qs, ts, ws, (4, 2, 24, 1), flag)


def test_long_banded_vs_reference(gpu):
    """Pairs of the long-interval workload's shape (scaled to 30-60 kb) against the compiled
    reference (native ISA entry, and its Singletrack entry): every field and the CIGAR
    through the per-pair hash."""
    from concurrent.futures import ThreadPoolExecutor
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    if ref.block != 64:
        pytest.skip("the device reproduces the AVX-512 padding lanes; this host's reference uses another block")
    ps = W.long_banded_set(6, seed=3, lmin=30_000, lmax=60_000, long_max=3_000)
    mat = oracle.anchorwave_matrix(-4)
    for flag, variant in ((0, 0), (ST, 2)):
        res = gpu.ksw_extd2_batch(ps.queries, ps.targets, mat, 4, 2, 24, 1, w=ps.band, flag=flag)

        def one(i):
            return int(ref.ksw_batch([ps.queries[i].tobytes()], [ps.targets[i].tobytes()], mat, 4, 2, 24, 1,
                                     w=ps.band[i], variant=variant, nthreads=1)["hash"][0])

        with ThreadPoolExecutor(len(ps)) as ex:
            cpu = list(ex.map(one, range(len(ps))))
        bad = [i for i, r in enumerate(res) if oracle.result_hash(r) != cpu[i]]
        assert not bad, f"flag {hex(flag)}: pairs {bad} differ"


def test_banded_repeatable_and_waves(gpu, restatement):
    """The same batch three times, the last split into traceback waves."""
    qs, ts, ws = _pairs(42, 30, 500, 4000, wfrac=(0.05, 0.3))
    mat = oracle.anchorwave_matrix(-4)
    exp = [restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w).key() for q, t, w in zip(qs, ts, ws)]
    try:
        for budget in (0, 0, 8 << 20):
            gpu.set_traceback_budget(budget)
            res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws)
            assert [r.key() for r in res] == exp, budget
    finally:
        gpu.set_traceback_budget(0)


@pytest.mark.parametrize("flag", [0, RIGHT, REV, SEMI])
def test_checkpointed_traceback(gpu, restatement, columns, flag):
    """Pairs whose traceback exceeds the budget: boundary columns on the first pass, then
    the walk recomputes strip groups from the last to the first.  A 2 MB budget splits each
    pair into several groups."""
    qs, ts, ws = _pairs(88 + flag, 10, 2000, 9000, wfrac=(0.05, 0.3))
    mat = oracle.anchorwave_matrix(-4)
    try:
        gpu.set_traceback_budget(2 << 20)
        res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=flag)
    finally:
        gpu.set_traceback_budget(0)
    for q, t, w, r in zip(qs, ts, ws, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w, flag=flag)
        assert r.key() == o.key(), (len(q), len(t), w)


def test_singletrack_beyond_budget_refused_alone(gpu, restatement):
    """A Singletrack pair whose two-track traceback exceeds the budget cannot be recomputed in
    strip groups: it alone is reported as the reference's allocation failure (reset result,
    zdropped = 1, no CIGAR); the other pairs of the batch are unaffected."""
    qs, ts, ws = _pairs(7, 6, 300, 900, wfrac=(0.1, 0.3))
    rng = np.random.default_rng(70)
    big_t = W.random_dna(rng, 9000)
    big_q = W.mutate(rng, big_t, 0.03, 0.005, 3.0)
    qs.insert(2, big_q), ts.insert(2, big_t), ws.insert(2, 2000)
    mat = oracle.anchorwave_matrix(-4)
    try:
        gpu.set_traceback_budget(4 << 20)  # the 9 kb pair needs ~40 MB of Singletrack traceback
        res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=ST)
    finally:
        gpu.set_traceback_budget(0)
    big = res[2]
    assert big.zdropped == 1 and big.n_cigar == 0 and big.score == oracle.KSW_NEG_INF
    for i, (q, t, w, r) in enumerate(zip(qs, ts, ws, res)):
        if i != 2:
            assert r.key() == restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w,
                                                   flag=ST).key()
