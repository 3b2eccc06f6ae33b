"""GPU tests of the serving loop (continuous batching): every result equals the standalone
call (alone vs in the mix), results are released strictly in id order, requests keep being
admitted while earlier micro-batches run, and a small HBM budget still completes the trace."""
import threading
import time

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

PEN = (4, 2, 24, 1)
WPEN = (4, 4, 2, 24, 1)


def _mix(seed, n):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        L = int(np.exp(rng.uniform(np.log(30), np.log(3000))))
        q, t = W.divergent_pair(rng, L, 0.01, 0.12, 4.0)
        if rng.random() < 0.1:
            q = q.copy()
            q[rng.integers(0, len(q), 2)] = 4
        kind = i % 7
        method = [0, 0, 1, 2, 3, 4, 5][kind]
        band = int(0.3 * min(len(q), len(t))) if kind == 1 else -1
        reqs.append((i, method, W.to_ascii(q), W.to_ascii(t), band))
    return reqs


def _standalone(gpu, wfa, method, q, t, band):
    from anchorwave_b200 import ksw2
    if method in (0, 1):
        qc, f1 = ksw2.encode(q)
        tc, f2 = ksw2.encode(t)
        fn = gpu.ksw_extd2_singletrack if method == 1 else gpu.ksw_extd2
        return fn(qc, tc, oracle.anchorwave_matrix(-4), *PEN, w=band, flag=f1 | f2).key()
    # routes 4 / 5: medium / low memory
    al = wfa.WfaAligner(*WPEN, singletrack=(method == 3), memory_mode=max(0, method - 3))
    st = al.align(t, q)
    ops, score = al.cigar() if st == 0 else ("", 0)
    al.close()
    return (st, score, ops)


def _drain(srv, n, timeout=120):
    out = []
    t0 = time.time()
    while len(out) < n and time.time() - t0 < timeout:
        out += srv.poll(256, wait_ms=50)
    return out


def test_results_identical_alone_and_in_the_mix(gpu):
    from anchorwave_b200 import serve, wfa
    reqs = _mix(11, 60)
    with serve.AlignmentServer(oracle.anchorwave_matrix(-4), *PEN, wfa_penalties=WPEN, slots=3,
                               max_batch=8) as srv:
        for rid, m, q, t, band in reqs:
            srv.submit(rid, m, q, t, band)
        got = _drain(srv, len(reqs))
        st = srv.stats()
    assert [g.id for g in got] == list(range(len(reqs)))
    assert st["micro_batches"] >= 4
    for g, (rid, m, q, t, band) in zip(got, reqs):
        alone = _standalone(gpu, wfa, m, q, t, band)
        assert (g.ksw if m in (0, 1) else g.wfa) == alone, (rid, m, len(q), len(t))


def test_ordered_release_behind_a_slow_request(gpu):
    from anchorwave_b200 import serve
    rng = np.random.default_rng(3)
    big_q, big_t = W.divergent_pair(rng, 12000, 0.05, 0.05, 4.0)
    with serve.AlignmentServer(oracle.anchorwave_matrix(-4), *PEN, wfa_penalties=WPEN, slots=2,
                               max_batch=1) as srv:
        srv.submit(0, 0, W.to_ascii(big_q), W.to_ascii(big_t))
        for i in range(1, 20):
            q, t = W.divergent_pair(rng, 100, 0.05, 0.05, 4.0)
            srv.submit(i, 0, W.to_ascii(q), W.to_ascii(t))
        got = _drain(srv, 20)
    assert [g.id for g in got] == list(range(20))


def test_continuous_arrivals_and_small_budget(gpu):
    """Requests arrive while earlier micro-batches run; a budget of a few traceback arenas
    forces admission waits; the whole trace still completes, in order, unchanged."""
    from anchorwave_b200 import serve, wfa
    reqs = _mix(29, 80)
    with serve.AlignmentServer(oracle.anchorwave_matrix(-4), *PEN, wfa_penalties=WPEN, slots=4, max_batch=4,
                               hbm_budget=96 << 20) as srv:
        def producer():
            for rid, m, q, t, band in reqs:
                srv.submit(rid, m, q, t, band)
                time.sleep(0.002)
        th = threading.Thread(target=producer)
        th.start()
        got = _drain(srv, len(reqs))
        th.join()
        st = srv.stats()
    assert [g.id for g in got] == list(range(len(reqs)))
    assert st["completed"] == len(reqs) and st["latency_p99_s"] >= st["latency_p50_s"] > 0
    for g, (rid, m, q, t, band) in list(zip(got, reqs))[::7]:
        assert (g.ksw if m in (0, 1) else g.wfa) == _standalone(gpu, wfa, m, q, t, band)


def _rows_key(rows_q, rows_d, score):
    """A rescue result as the server returns it: the rows as an M/I/D CIGAR and the score."""
    cig, i, n = [], 0, len(rows_q)
    while i < n:
        op = 2 if rows_q[i] == "-" else 1 if rows_d[i] == "-" else 0
        j = i + 1
        while j < n and (2 if rows_q[j] == "-" else 1 if rows_d[j] == "-" else 0) == op:
            j += 1
        cig.append(((j - i) << 4) | op)
        i = j
    return score, tuple(cig)


def _rescue_standalone(method, q, t, band, band_max, window):
    from anchorwave_b200 import ksw2
    pen = (-4, -4, -2, -24, -1)
    if method == 6:
        r = ksw2.align_score_certified_ksw2_batch([(q.decode(), t.decode())], band, band_max, *pen)[0]
        status = {ksw2.CERT_COMPLETED: 0, ksw2.CERT_TIME_LIMIT: 1, ksw2.CERT_NOT_CERTIFIED: 2, ksw2.CERT_FAILED: 3}
        rq, rd = ((r.alignment_q, r.alignment_d) if r.alignment_q else
                  (r.best_effort_query_alignment, r.best_effort_reference_alignment))
        return status[r.status], _rows_key(rq, rd, r.score)
    s, rq, rd = ksw2.align_sliding_window_batch([(q.decode(), t.decode())], window, 0, *pen)[0]
    return 0, _rows_key(rq, rd, s)


def test_rescue_routes_alone_and_in_the_mix(gpu):
    """Score-certified KSW2 and sliding-window requests (the selector's rescue outcomes) go
    through the server beside the other engines; each result equals the standalone batch
    entry's (status, rows as CIGAR, re-scored score)."""
    from anchorwave_b200 import serve
    rng = np.random.default_rng(41)
    reqs = []
    for i in range(36):
        L = int(rng.integers(200, 2500))
        q, t = W.divergent_pair(rng, L, 0.02, 0.12, 4.0)
        if i % 4 == 0 and len(q) > 400:
            at = int(rng.integers(0, len(q) - 300))
            q = np.concatenate([q[:at], q[at + int(rng.integers(40, 250)):]])
        method = [6, 7, 0, 6, 7, 2][i % 6]
        band, band_max, window = (16, 600, 0) if method == 6 else (-1, -1, 300) if method == 7 else (-1, -1, 0)
        reqs.append((i, method, W.to_ascii(q), W.to_ascii(t), band, band_max, window))
    with serve.AlignmentServer(oracle.anchorwave_matrix(-4), *PEN, wfa_penalties=WPEN, slots=3,
                               max_batch=5) as srv:
        for rid, m, q, t, b, bm, w in reqs:
            srv.submit(rid, m, q, t, band=b, band_max=bm, window=w)
        got = _drain(srv, len(reqs))
    assert [g.id for g in got] == list(range(len(reqs)))
    for g, (rid, m, q, t, b, bm, w) in zip(got, reqs):
        if m in (6, 7):
            st, key = _rescue_standalone(m, q, t, b, bm, w)
            assert g.status == st and (g.ksw[8], g.ksw[12]) == key, (rid, m)
    assert {g.method for g in got} == {0, 2, 6, 7}


def test_selector_routes_reproduced(gpu):
    """Intervals routed by AnchorWave's own selector (the routing front end) are served with
    exactly the chosen engine and parameters, and each result equals that engine's standalone
    result."""
    try:
        from anchorwave_b200 import route
    except ImportError as e:
        pytest.skip(str(e))
    from anchorwave_b200 import serve, wfa
    reqs = W.serving_trace(48, seed=12, lmax=20_000)
    routes = route.route_intervals([(r.query, r.target) for r in reqs])
    with serve.AlignmentServer(oracle.anchorwave_matrix(-4), *PEN, wfa_penalties=WPEN, slots=2,
                               max_batch=8) as srv:
        for r, rt in zip(reqs, routes):
            srv.submit(r.id, rt.method, r.query, r.target, band=rt.band, band_max=rt.band_max, window=rt.window,
                       predicted_bytes=rt.predicted_bytes)
        got = _drain(srv, len(reqs))
    assert [g.id for g in got] == [r.id for r in reqs]
    for g, r, rt in zip(got, reqs, routes):
        assert g.method == rt.method
        if rt.method in (6, 7):
            st, key = _rescue_standalone(rt.method, r.query, r.target, rt.band, rt.band_max, rt.window)
            assert g.status == st and (g.ksw[8], g.ksw[12]) == key
        else:
            alone = _standalone(gpu, wfa, rt.method, r.query, r.target, rt.band)
            assert (g.ksw if rt.method in (0, 1) else g.wfa) == alone, (r.id, rt)
