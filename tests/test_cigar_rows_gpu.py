"""Gapped rows decoded on the device (aw_cigar_rows_batch) from the GPU's KSW2 CIGARs against
the compiled reference's minimap2AlignmentWithArena (alignSlidingWindow.cpp:241-332: its own
ksw_extd2 call and the CIGAR decoding of :307-324) on the same intervals, for results with
mismatches, long indels, N bases and lowercase letters (the rows keep the caller's
characters), and the rejected inputs."""
import numpy as np
import pytest

from anchorwave_b200 import ksw2
from anchorwave_b200._lib import AwError
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_rows_match_compiled_reference(gpu, reference):
    rng = np.random.default_rng(12)
    qs, ts = [], []
    for i in range(64):
        t = W.random_dna(rng, int(rng.integers(1, 6000)))
        q = W.mutate(rng, t, 0.05, 0.02, 6.0)
        if len(q) == 0:
            q = t[:1].copy()
        dq, dd = W.to_ascii(q).decode(), W.to_ascii(t).decode()
        if i % 4 == 1:
            dq = dq.lower()
        if i % 5 == 2:
            dd = "N" + dd[1:]
        qs.append(dq)
        ts.append(dd)
    codes = [(ksw2.encode(q), ksw2.encode(t)) for q, t in zip(qs, ts)]
    res = []
    for (qc, f1), (tc, f2) in codes:
        res.append(ksw2.ksw_extd2(qc, tc, ksw2.anchorwave_matrix(-4), 4, 2, 24, 1, flag=f1 | f2))
    rows = ksw2.cigar_rows_batch([r.cigar for r in res], qs, ts)
    for q, t, r, (rq, rd) in zip(qs, ts, res, rows):
        score, eq, ed = reference.minimap2_rows(q, t, (-4, -4, -2, -24, -1))
        assert score == r.score
        assert (rq, rd) == (eq, ed)
        assert rq.replace("-", "") == q and rd.replace("-", "") == t


def test_rows_reject_bad_cigars(gpu):
    with pytest.raises(AwError):
        ksw2.cigar_rows_batch([[(5 << 4) | 4]], ["ACGTA"], ["ACGTA"])  # soft clip: not a KSW2 op
    with pytest.raises(AwError):
        ksw2.cigar_rows_batch([[(6 << 4) | 0]], ["ACGTA"], ["ACGTAC"])  # M runs past the query
    assert ksw2.cigar_rows_batch([[]], [""], [""]) == [("", "")]
