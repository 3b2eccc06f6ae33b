"""GPU cooperative stop (the deadline AnchorWave installs with ksw_set_progress_callback,
alignSlidingWindow.cpp:593-640, minimap2/ksw2_progress.c) through the C ABI.

* The deterministic form (stop at the first probed anti-diagonal >= r) is bit-exact
  against the oracle restatement's stop hook, which is itself pinned against the compiled
  reference: every ksw_extz_t field, the partial traceback of a stopped pair included.
* The wall-clock form stops nothing when the deadline is far, stops everything when it
  has passed, and in between every pair is either stopped (score KSW_NEG_INF, no CIGAR)
  or identical to the undisturbed run, on all three kernels (full-width strips, banded
  strips, anti-diagonal)."""
import threading
import time

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

SCORE_ONLY, ST = 0x01, 0x1000
NEG_INF = -0x40000000


def _pairs(seed, n, lmin, lmax, dmax=0.1):
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for _ in range(n):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        q, t = W.divergent_pair(rng, L, 0.01, dmax, 4.0)
        qs.append(q)
        ts.append(t)
    return qs, ts


@pytest.fixture
def no_stop(gpu):
    yield
    gpu.set_deadline(0)
    gpu.set_stop_antidiagonal(256, -1)


@pytest.mark.parametrize("flag", [0, SCORE_ONLY, ST])
@pytest.mark.parametrize("stop_at", [0, 256, 700, 2000, 100000])
def test_stop_antidiagonal_vs_restatement(gpu, restatement, no_stop, flag, stop_at):
    qs, ts = _pairs(stop_at + flag, 24, 50, 2500)
    rng = np.random.default_rng(9)
    ws = [int(rng.integers(20, 400)) if i % 2 else -1 for i in range(len(qs))]
    mat = oracle.anchorwave_matrix(-4)
    gpu.set_stop_antidiagonal(256, stop_at)
    res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=flag)
    gpu.set_stop_antidiagonal(256, -1)
    for q, t, w, r in zip(qs, ts, ws, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, w=w, flag=flag,
                                  stop_interval=256, stop_at=stop_at)
        assert r.key() == o.key(), (len(q), len(t), w, stop_at)
    if stop_at == 0:
        assert all(r.stopped for r in res)


def test_stop_antidiagonal_vs_reference(gpu, reference, no_stop):
    """Stopped pairs against the compiled reference with its progress hook."""
    qs, ts = _pairs(4, 8, 300, 1500)
    mat = oracle.anchorwave_matrix(-4)
    for stop_at in (256, 1024):
        gpu.set_stop_antidiagonal(256, stop_at)
        res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1)
        gpu.set_stop_antidiagonal(256, -1)
        for q, t, r in zip(qs, ts, res):
            o = reference.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, stop_interval=256, stop_at=stop_at)
            assert r.key() == o.key(), (len(q), len(t), stop_at)


def _mixed_batch():
    """Pairs for all three routes: full width (strip kernel), banded (banded strip kernel)
    and z-drop (anti-diagonal kernel)."""
    qs, ts = _pairs(31, 30, 200, 6000)
    ws = [-1 if i % 3 == 0 else int(0.1 * max(len(q), len(t))) + 5 for i, (q, t) in enumerate(zip(qs, ts))]
    return qs, ts, ws


@pytest.mark.parametrize("flag", [0, SCORE_ONLY, ST])
def test_far_deadline_changes_nothing(gpu, no_stop, flag):
    qs, ts, ws = _mixed_batch()
    mat = oracle.anchorwave_matrix(-4)
    ref = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=flag)
    refz = gpu.ksw_extd2_batch(qs[:6], ts[:6], mat, 4, 2, 24, 1, w=ws[:6], zdrop=400, flag=flag)
    with gpu.deadline(600.0):
        res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=flag)
        resz = gpu.ksw_extd2_batch(qs[:6], ts[:6], mat, 4, 2, 24, 1, w=ws[:6], zdrop=400, flag=flag)
    assert [r.key() for r in res] == [r.key() for r in ref]
    assert [r.key() for r in resz] == [r.key() for r in refz]
    assert not any(r.stopped for r in res + resz)


@pytest.mark.parametrize("flag", [0, SCORE_ONLY, ST])
def test_passed_deadline_stops_every_pair(gpu, no_stop, flag):
    qs, ts, ws = _mixed_batch()
    mat = oracle.anchorwave_matrix(-4)
    gpu.set_deadline(1e-9)
    time.sleep(0.01)
    res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, w=ws, flag=flag)
    resz = gpu.ksw_extd2_batch(qs[:6], ts[:6], mat, 4, 2, 24, 1, w=ws[:6], zdrop=400, flag=flag)
    single = gpu.ksw_extd2(qs[1], ts[1], mat, 4, 2, 24, 1, w=ws[1], flag=flag)
    gpu.set_deadline(0)
    for r in res + resz + [single]:
        assert r.stopped == 1 and r.score == NEG_INF and r.n_cigar == 0
    # cleared: the next call runs to the end
    again = gpu.ksw_extd2_batch(qs[:3], ts[:3], mat, 4, 2, 24, 1, w=ws[:3], flag=flag)
    assert not any(r.stopped for r in again)


@pytest.mark.parametrize("kind", ["full", "banded"])
def test_deadline_mid_batch(gpu, no_stop, kind):
    """A deadline that passes while the batch runs: each pair is either stopped or
    identical to the undisturbed run, and the call returns soon after the deadline."""
    rng = np.random.default_rng(5)
    qs, ts = [], []
    for _ in range(96):
        q, t = W.divergent_pair(rng, int(rng.integers(8000, 16000)), 0.01, 0.05, 4.0)
        qs.append(q)
        ts.append(t)
    ws = [-1] * len(qs) if kind == "full" else [int(0.2 * max(len(q), len(t))) for q, t in zip(qs, ts)]
    mat = oracle.anchorwave_matrix(-4)
    call = gpu.BatchCall(qs, ts, mat, 4, 2, 24, 1, w=ws)
    call.run()
    call.results()
    t0 = time.perf_counter()
    call.run()
    full_s = time.perf_counter() - t0
    ref = call.results()
    stopped = 0
    for frac in (0.5, 0.2):
        with gpu.deadline(full_s * frac):
            t0 = time.perf_counter()
            call.run()
            took = time.perf_counter() - t0
        res = call.results()
        for r, o in zip(res, ref):
            if r.stopped:
                stopped += 1
                assert r.score == NEG_INF and r.n_cigar == 0
            else:
                assert r.key() == o.key()
        assert took < full_s * frac + 0.5 + 0.5 * full_s, (took, full_s)
    assert stopped > 0, full_s


def test_deadline_is_per_thread(gpu, no_stop):
    """A passed deadline on this thread leaves another thread's calls alone."""
    qs, ts = _pairs(8, 6, 500, 3000)
    mat = oracle.anchorwave_matrix(-4)
    gpu.set_deadline(1e-9)
    out = {}

    def worker():
        out["res"] = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1)
        gpu.release_thread_buffers()

    th = threading.Thread(target=worker)
    th.start()
    th.join()
    mine = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1)
    gpu.set_deadline(0)
    assert not any(r.stopped for r in out["res"])
    assert all(r.stopped for r in mine)
