"""GPU parity of ksw_extd2_singletrack_sse_gpu (the Singletrack entry of AnchorWave builds
without AVX2, minimap2/ksw2_singletrack.cpp:202-626) through the C ABI: every ksw_extz_t field
and the CIGAR against the restatement (16-byte blocks, Singletrack) and the compiled
reference's SSE Singletrack entry."""
import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

FLAGS = [0, oracle.KSW_EZ_SEMIGLOBAL_END, oracle.KSW_EZ_EXTZ_ONLY, oracle.KSW_EZ_REV_CIGAR,
         oracle.KSW_EZ_SCORE_ONLY, oracle.KSW_EZ_APPROX_MAX | oracle.KSW_EZ_APPROX_DROP,
         oracle.KSW_EZ_RIGHT | oracle.KSW_EZ_GENERIC_SC]
PEN = [(4, 2, 24, 1), (8, 2, 75, 1), (6, 1, 20, 0), (2, 3, 30, 1)]


def _cases(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for it in range(n):
        L = int(np.exp(rng.uniform(np.log(1), np.log(2500))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.25, 4.0)
        if it % 6 == 5:
            q = q.copy()
            q[rng.integers(0, len(q), 3)] = 4
        w = -1 if it % 2 == 0 else int(rng.integers(0, max(1, L // 3)))
        out.append((q, t, FLAGS[it % len(FLAGS)], w, -1 if it % 3 else 100, PEN[it % len(PEN)]))
    return out


def test_sse_singletrack_vs_oracle(gpu, restatement):
    from anchorwave_b200 import ksw2
    mat = oracle.anchorwave_matrix(-4)
    for i, (q, t, flag, w, zdrop, pen) in enumerate(_cases(3, 120)):
        g = ksw2.ksw_extd2_singletrack_sse(q, t, mat, *pen, w=w, zdrop=zdrop, flag=flag)
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w, zdrop=zdrop,
                                  flag=flag | oracle.KSW_EZ_SINGLETRACK, block=16)
        assert g.key() == o.key(), (i, len(q), len(t), w, hex(flag), pen)


def test_sse_singletrack_vs_reference_and_batch(gpu):
    from anchorwave_b200 import ksw2
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    mat = oracle.anchorwave_matrix(-4)
    cases = [c for c in _cases(9, 60) if c[2] == 0 and c[4] == -1 and c[5] == PEN[0]]
    for q, t, flag, w, zdrop, pen in cases:
        g = ksw2.ksw_extd2_singletrack_sse(q, t, mat, *pen, w=w)
        r = ref.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w, variant=3)
        assert g.key() == r.key(), (len(q), len(t), w)
    # the batch entry with the flags gives the same results as the single calls
    qs = [c[0] for c in cases]
    ts = [c[1] for c in cases]
    ws = [c[3] for c in cases]
    got = ksw2.ksw_extd2_batch(qs, ts, mat, *PEN[0], w=ws,
                               flag=oracle.KSW_EZ_SINGLETRACK | 0x4000)
    for q, t, w, b in zip(qs, ts, ws, got):
        assert b.key() == ksw2.ksw_extd2_singletrack_sse(q, t, mat, *PEN[0], w=w).key()
