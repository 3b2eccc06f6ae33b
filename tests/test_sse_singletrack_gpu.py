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


def _band_cases(seed, n):
    """Pairs of 300 bp-12 kb that take the banded strip kernel: no z-drop, every flag it
    serves, bands from empty-before-the-end to full width, and low-complexity pairs."""
    rng = np.random.default_rng(seed)
    flags = [0, oracle.KSW_EZ_SEMIGLOBAL_END, oracle.KSW_EZ_SCORE_ONLY, oracle.KSW_EZ_REV_CIGAR,
             oracle.KSW_EZ_RIGHT | oracle.KSW_EZ_GENERIC_SC,
             oracle.KSW_EZ_SEMIGLOBAL_END | oracle.KSW_EZ_SCORE_ONLY]
    out = []
    for it in range(n):
        L = int(np.exp(rng.uniform(np.log(300), np.log(12000))))
        if it % 5 == 4:
            unit = W.random_dna(rng, int(rng.integers(1, 5)))
            t = np.tile(unit, L // len(unit) + 1)[:L]
            q = t[: max(1, L - int(rng.integers(0, 40)))].copy()
        else:
            q, t = W.divergent_pair(rng, L, 0.01, 0.2, 4.0)
        w = [-1, L // 10, L // 3, 0, 7][it % 5]
        out.append((q, t, flags[it % len(flags)], w, PEN[it % 2]))
    return out


def test_sse_singletrack_banded_kernel_vs_oracle(gpu, restatement):
    """The SSE Singletrack entry's pairs run on the banded strip kernel (16-byte blocks, the
    strict end rules, reconstruction whatever the flags): identical to the restatement."""
    from anchorwave_b200 import ksw2
    mat = oracle.anchorwave_matrix(-4)
    cases = _band_cases(21, 36)
    for flag in sorted({c[2] for c in cases}):
        for pen in PEN[:2]:
            sub = [c for c in cases if c[2] == flag and c[4] == pen]
            if not sub:
                continue
            plan = ksw2.KswPlan([c[0] for c in sub], [c[1] for c in sub], mat, *pen,
                                w=[c[3] for c in sub], flag=flag | oracle.KSW_EZ_SINGLETRACK | 0x4000)
            assert plan.routes()["exact"] == 0, (hex(flag), plan.routes())
            plan.upload()
            plan.execute()
            got = plan.download()
            plan.close()
            for (q, t, _, w, _), g in zip(sub, got):
                o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w,
                                          flag=flag | oracle.KSW_EZ_SINGLETRACK, block=16)
                assert g.key() == o.key(), (len(q), len(t), w, hex(flag), pen)
