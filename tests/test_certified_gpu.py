"""Score-certified KSW2 (alignScoreCertifiedKsw2, alignSlidingWindow.cpp:1197-1400) on the
GPU, one interval at a time and batched, against a restatement of the same procedure whose
DP passes run on the oracle: every field of the result and the alignment rows."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import ksw2
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
PEN = (-4, -4, -2, -24, -1)  # AnchorWave's mismatch and gap penalties (negative)


def _restated(restatement, dq, dd, initial, maximum, pen):
    """The reference procedure step by step, with the oracle's ksw_extd2 for every DP."""
    mis, o1, e1, o2, e2 = pen
    mat = ksw2.anchorwave_matrix(mis)
    r = ksw2.CertifiedResult()
    if min(len(dq), len(dd)) == 0:
        r.alignment_q = dq if dq else "-" * len(dd)
        r.alignment_d = dd if dd else "-" * len(dq)
        ln = max(len(dq), len(dd))
        r.score = r.optimal_score = max(o1 + e1 * ln, o2 + e2 * ln)
        r.final_band_width, r.traceback_attempts, r.status = 0, 1, ksw2.CERT_COMPLETED
        return r
    diff = abs(len(dq) - len(dd))
    if initial < 0 or maximum < 0 or maximum < diff:
        r.status = ksw2.CERT_NOT_CERTIFIED
        return r
    qs, f1 = ksw2.encode(dq)
    ts, f2 = ksw2.encode(dd)

    def dp(w, flag):
        return restatement.ksw_extd2(qs.tobytes(), ts.tobytes(), mat, -o1, -e1, -o2, -e2, w=w, flag=f1 | f2 | flag)

    r.optimal_score = dp(-1, ksw2.KSW_EZ_SCORE_ONLY).score
    if r.optimal_score == ksw2.KSW_NEG_INF:
        r.status = ksw2.CERT_FAILED
        return r
    max_band = min(max(len(dq), len(dd)), maximum)

    def attempt(band):
        res = dp(band, 0)
        s, aq, ad = ksw2._banded_rows(res, dq, dd, pen)
        valid = len(aq) == len(ad) and aq.replace("-", "") == dq and ad.replace("-", "") == dd
        return s, aq, ad, valid

    requested = max(diff, max(1, initial))
    doubled = requested * 2
    band = min(max_band, max(requested, doubled))
    while diff <= band <= max_band:
        r.traceback_attempts += 1
        s, aq, ad, valid = attempt(band)
        if s == r.optimal_score and valid:
            r.score, r.final_band_width, r.alignment_q, r.alignment_d = s, band, aq, ad
            r.status = ksw2.CERT_COMPLETED
            return r
        if valid and (not r.best_effort_query_alignment or s > r.score):
            r.score, r.best_effort_query_alignment, r.best_effort_reference_alignment = s, aq, ad
        if band == max_band:
            break
        nxt = min(max_band, max(band + 1, band * 2))
        if nxt <= band:
            break
        band = nxt
    if requested < min(max_band, doubled):
        r.traceback_attempts += 1
        s, aq, ad, valid = attempt(requested)
        if s == r.optimal_score and valid:
            r.score, r.final_band_width, r.alignment_q, r.alignment_d = s, requested, aq, ad
            r.status = ksw2.CERT_COMPLETED
            return r
        if valid and (not r.best_effort_query_alignment or s > r.score):
            r.score, r.best_effort_query_alignment, r.best_effort_reference_alignment = s, aq, ad
    r.final_band_width = band
    r.status = ksw2.CERT_NOT_CERTIFIED
    return r


def _intervals(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(rng.integers(150, 3000))
        t = W.random_dna(rng, L)
        if i % 4 == 0:
            # a long deletion: small bands cannot hold the optimal path
            q = W.mutate(rng, t, 0.03, 0.005, 3.0)
            at = int(rng.integers(0, max(1, len(q) - 400)))
            q = np.concatenate([q[:at], q[at + int(rng.integers(50, 300)):]])
        elif i % 4 == 1:
            q = W.mutate(rng, t, 0.1, 0.03, 4.0)
        else:
            q = W.mutate(rng, t, 0.02, 0.005, 3.0)
        dq, dd = W.to_ascii(q).decode(), W.to_ascii(t).decode()
        if i % 7 == 3:
            dq = dq[:10] + "N" + dq[11:]
        out.append((dq, dd))
    out.append(("", "ACGTACGT"))
    out.append(("ACGT" * 50, "ACGT" * 20))  # length difference beyond the largest band below
    return out


@pytest.mark.parametrize("initial,maximum", [(16, 2000), (100, 400), (1, 64)])
def test_certified_batch_vs_restatement(gpu, restatement, initial, maximum):
    pairs = _intervals(initial + maximum, 24)
    got = ksw2.align_score_certified_ksw2_batch(pairs, initial, maximum, *PEN)
    statuses = set()
    for (dq, dd), g in zip(pairs, got):
        exp = _restated(restatement, dq, dd, initial, maximum, PEN)
        assert g == exp, (len(dq), len(dd), g.status, exp.status)
        statuses.add(g.status)
    assert ksw2.CERT_COMPLETED in statuses
    if initial <= 16:
        # a 32-column first band cannot hold the 50-300 bp deletions: some intervals widen
        assert max(g.traceback_attempts for g in got) >= 2


def test_certified_single_equals_batch(gpu):
    pairs = _intervals(5, 8)
    batch = ksw2.align_score_certified_ksw2_batch(pairs, 32, 1000, *PEN)
    for (dq, dd), b in zip(pairs, batch):
        assert ksw2.align_score_certified_ksw2(dq, dd, 32, 1000, *PEN) == b


def test_certified_under_passed_deadline(gpu):
    """A deadline that has already passed stops the score pass: TimeLimit, no rows."""
    pairs = _intervals(9, 4)[:4]
    got = ksw2.align_score_certified_ksw2_batch(pairs, 16, 1000, *PEN, maximum_runtime_seconds=1e-9)
    assert all(g.status == ksw2.CERT_TIME_LIMIT and not g.alignment_q for g in got)
