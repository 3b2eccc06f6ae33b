"""Sliding-window semiglobal alignment (alignSlidingWindow, alignSlidingWindow.cpp:457-590) on
the GPU, one interval at a time and batched (window i of every interval in one call), against
the same procedure with the oracle's ksw_extd2 for every window: the score and both rows."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import ksw2
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
PEN = (0, -4, -4, -2, -24, -1)  # matching score, mismatch, gap penalties (AnchorWave's, negative)


def _restated(restatement, dq, dd, win, pen):
    match, mis, o1, e1, o2, e2 = pen

    def dp(q, d, mis_, o1_, e1_, o2_, e2_, flag):
        qs, f1 = ksw2.encode(q)
        ts, f2 = ksw2.encode(d)
        return restatement.ksw_extd2(qs.tobytes(), ts.tobytes(), ksw2.anchorwave_matrix(mis_), -o1_, -e1_, -o2_, -e2_,
                                     flag=f1 | f2 | flag)

    aq, ad = "", ""
    qs_, ds_ = 1, 1
    if (len(dd) / win) * (len(dq) / win) <= 1:
        r = dp(dq, dd, mis, o1, e1, o2, e2, 0)
        a, b, _, _ = ksw2.decode_cigar(r.cigar, dq, dd)
        aq, ad = a, b
        qs_, ds_ = len(dq) + 1, len(dd) + 1
    else:
        wp = ((mis + match, o1 + match, e1 + match, o2 + match, e2 + match) if e2 + match < 0 else
              (mis + match - 1, o1 + match - 1, e1 + match - 1, o2 + match - 1, -1))
        while ds_ <= len(dd) and qs_ <= len(dq):
            qw = dq[qs_ - 1:min(qs_ + win, len(dq))]
            dw = dd[ds_ - 1:min(ds_ + win, len(dd))]
            r = dp(qw, dw, *wp, ksw2.KSW_EZ_SEMIGLOBAL_END)
            if r.mqe > r.mte:
                et, eq = r.mqe_t + 1, len(qw)
            else:
                et, eq = len(dw), r.mte_q + 1
            a, b, _, _ = ksw2.decode_cigar(r.cigar, qw, dw)
            aq += a
            ad += b
            qs_ += eq
            ds_ += et
    if len(dd) - ds_ >= 0:
        aq += "-" * (len(dd) - ds_ + 1)
        ad += dd[ds_ - 1:]
    if len(dq) - qs_ >= 0:
        aq += dq[qs_ - 1:]
        ad += "-" * (len(dq) - qs_ + 1)
    return ksw2.score_gapped_two_piece_affine(aq, ad, mis, o1, e1, o2, e2), aq, ad


def _intervals(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        t = W.random_dna(rng, int(rng.integers(100, 4000)))
        q = W.mutate(rng, t, 0.05, 0.01, 4.0)
        if i % 3 == 0 and len(q) > 600:
            at = int(rng.integers(0, len(q) - 500))
            q = np.concatenate([q[:at], q[at + int(rng.integers(20, 400)):]])
        dq, dd = W.to_ascii(q).decode(), W.to_ascii(t).decode()
        if i % 5 == 2:
            dd = dd[:7] + "N" + dd[8:]
        out.append((dq, dd))
    return out


@pytest.mark.parametrize("win", [150, 400, 2000])
def test_sliding_window_batch_vs_restatement(gpu, restatement, win):
    pairs = _intervals(win, 20)
    got = ksw2.align_sliding_window_batch(pairs, win, *PEN)
    for (dq, dd), g in zip(pairs, got):
        exp = _restated(restatement, dq, dd, win, PEN)
        assert g == exp, (len(dq), len(dd), win)
        assert g[1].replace("-", "") == dq and g[2].replace("-", "") == dd


def test_sliding_window_single_equals_batch(gpu):
    pairs = _intervals(3, 6)
    batch = ksw2.align_sliding_window_batch(pairs, 300, *PEN)
    for (dq, dd), b in zip(pairs, batch):
        assert ksw2.align_sliding_window(dq, dd, 300, *PEN) == b
