"""Score-certified KSW2 (alignScoreCertifiedKsw2, alignSlidingWindow.cpp:1197-1400) on the
GPU through aw_align_score_certified_batch, one interval at a time and batched, against the
compiled reference's own alignScoreCertifiedKsw2 (oracle/ref_rescue_shim.cpp, no selection
plan, no deadline) on the same intervals: every field of the result, the certified rows and
the best-effort rows."""
import numpy as np
import pytest

from anchorwave_b200 import ksw2
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
PEN = (-4, -4, -2, -24, -1)  # AnchorWave's mismatch and gap penalties (negative)
STATUS = {0: ksw2.CERT_COMPLETED, 1: ksw2.CERT_TIME_LIMIT, 2: ksw2.CERT_NOT_CERTIFIED, 3: ksw2.CERT_FAILED}


def _reference_result(reference, dq, dd, initial, maximum):
    r = reference.score_certified(dq, dd, initial, maximum, PEN)
    return ksw2.CertifiedResult(status=STATUS[r["status"]], score=r["score"], optimal_score=r["optimal_score"],
                                final_band_width=r["final_band_width"], traceback_attempts=r["traceback_attempts"],
                                best_effort_query_alignment=r["best_effort_q"],
                                best_effort_reference_alignment=r["best_effort_d"],
                                alignment_q=r["alignment_q"], alignment_d=r["alignment_d"])


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
def test_certified_batch_vs_compiled_reference(gpu, reference, initial, maximum):
    pairs = _intervals(initial + maximum, 24)
    got = ksw2.align_score_certified_ksw2_batch(pairs, initial, maximum, *PEN)
    statuses = set()
    for (dq, dd), g in zip(pairs, got):
        exp = _reference_result(reference, dq, dd, initial, maximum)
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
