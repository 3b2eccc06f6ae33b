/*
 * wfa_oracle.c -- TEST INFRASTRUCTURE (oracle).  Plain-C restatement of the
 * WFA2-lib gap-affine-2p end-to-end aligner exactly as AnchorWave configures it
 * (src/myImportandFunction/WfaAlignment.cpp:143-170: match 0, high memory,
 * no heuristic, full CIGAR; standard or Singletrack traceback).  Used only by
 * tests/ to check the CUDA WFA path; pinned against the compiled WFA2-lib
 * (oracle/_ref) and the golden vectors in tests/golden/wfa_golden.json.
 *
 * Restated (WFA2-lib file:line):
 *   unidirectional loop       wavefront/wavefront_unialign.c:262-293
 *   input fetch               wavefront/wavefront_compute.c:325-371
 *   limits (null wf lo=1,hi=-1) wavefront/wavefront_compute.c:56-105, wavefront.c:110-117
 *   output allocation rule    wavefront/wavefront_compute.c:459-572
 *   affine-2p kernel          wavefront/wavefront_compute_affine2p.c:45-106
 *   trim ends                 wavefront/wavefront_compute.c:654-690
 *   extend + end2end stop     wavefront/wavefront_extend.c:86-121,
 *                             wavefront/wavefront_termination.c:37-60
 *   backtrace (piggyback ties) wavefront/wavefront_backtrace.c:41-60, :321-530
 *   Singletrack backtrace     wavefront/wavefront_backtrace.c:587-762
 * Every wavefront value outside its trimmed [lo, hi] reads as NULL, which is
 * what the reference's init_ends NULL padding makes it.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

#define WO_NULL (INT32_MIN / 2)

typedef struct {
    int lo, hi;      /* trimmed range; lo > hi means null */
    int base;        /* off[k - base] */
    int32_t *off;
} wo_wf;

typedef struct {
    wo_wf *M, *I1, *D1, *I2, *D2; /* NULL pointer: no wavefront for that score */
} wo_score;

static int32_t wo_get(const wo_wf *w, int k) {
    if (!w || w->lo > w->hi || k < w->lo || k > w->hi) return WO_NULL;
    return w->off[k - w->base];
}
static int wo_isnull(const wo_wf *w) { return !w || w->lo > w->hi; }
static __thread long long wo_ints_allocated = 0;
/* Offsets allocated by the last oracle_wfa_align call on this thread (sizing aid). */
long long oracle_wfa_last_ints(void) { return wo_ints_allocated; }
static wo_wf *wo_new(int lo, int hi) {
    wo_wf *w = (wo_wf *)malloc(sizeof(wo_wf));
    wo_ints_allocated += hi - lo + 1 > 0 ? hi - lo + 1 : 1;
    w->lo = lo, w->hi = hi, w->base = lo;
    w->off = (int32_t *)malloc(sizeof(int32_t) * (size_t)(hi - lo + 1 > 0 ? hi - lo + 1 : 1));
    return w;
}
static void wo_free(wo_wf *w) {
    if (w) free(w->off), free(w);
}
static void wo_trim(wo_wf *w, int plen, int tlen) {
    int k;
    for (k = w->hi; k >= w->lo; --k) {
        const int32_t o = w->off[k - w->base];
        const uint32_t h = (uint32_t)o, v = (uint32_t)(o - k);
        if (h <= (uint32_t)tlen && v <= (uint32_t)plen) break;
    }
    w->hi = k;
    for (k = w->lo; k <= w->hi; ++k) {
        const int32_t o = w->off[k - w->base];
        const uint32_t h = (uint32_t)o, v = (uint32_t)(o - k);
        if (h <= (uint32_t)tlen && v <= (uint32_t)plen) break;
    }
    w->lo = k;
}
static int32_t mx(int32_t a, int32_t b) { return a > b ? a : b; }

/*
 * pattern = reference (length plen), text = query (length tlen).  Returns the
 * WF status (0 = completed, -300 = unattainable Singletrack traceback); on
 * success *score is the classic score (-penalty) and ops[0..*n_ops) the CIGAR
 * operations (M match, X mismatch, I text-only, D pattern-only).
 */
int oracle_wfa_align(const char *pattern, int plen, const char *text, int tlen, int x, int o1, int e1,
                     int o2, int e2, int singletrack, int *score_out, char *ops, int ops_cap, int *n_ops) {
    *score_out = 0, *n_ops = 0;
    wo_ints_allocated = 0;
    const int scope = (o1 + e1 > o2 + e2 ? o1 + e1 : o2 + e2);
    const int max_score_scope = (scope > x ? scope : x) + 1;
    int cap = 1024, s = 0, num_null = 0;
    wo_score *W = (wo_score *)calloc((size_t)cap, sizeof(wo_score));
    W[0].M = wo_new(0, 0);
    W[0].M->off[0] = 0;
    const int k_end = tlen - plen;
    int status = 0, end_score = -1;
    for (;;) {
        /* extend + termination */
        wo_wf *m = W[s].M;
        if (m) {
            for (int k = m->lo; k <= m->hi; ++k) {
                int32_t o = m->off[k - m->base];
                if (o == WO_NULL) continue;
                int h = o, v = o - k;
                while (v < plen && h < tlen && pattern[v] == text[h]) ++v, ++h;
                m->off[k - m->base] = h;
            }
            if (!(m->lo > k_end || k_end > m->hi) && m->off[k_end - m->base] >= tlen) {
                end_score = s;
                break;
            }
        } else if (num_null > max_score_scope) {
            status = -3; /* end unreachable: cannot happen end-to-end without heuristics */
            break;
        }
        /* compute s+1 */
        ++s;
        if (s >= cap) {
            W = (wo_score *)realloc(W, sizeof(wo_score) * (size_t)cap * 2);
            memset(W + cap, 0, sizeof(wo_score) * (size_t)cap);
            cap *= 2;
        }
        const int sm = s - x, so1 = s - o1 - e1, se1 = s - e1, so2 = s - o2 - e2, se2 = s - e2;
        wo_wf *m_misms = sm >= 0 ? W[sm].M : 0, *m_open1 = so1 >= 0 ? W[so1].M : 0;
        wo_wf *i1 = se1 >= 0 ? W[se1].I1 : 0, *d1 = se1 >= 0 ? W[se1].D1 : 0;
        wo_wf *m_open2 = so2 >= 0 ? W[so2].M : 0;
        wo_wf *i2 = se2 >= 0 ? W[se2].I2 : 0, *d2 = se2 >= 0 ? W[se2].D2 : 0;
        if (wo_isnull(m_misms)) m_misms = 0;
        if (wo_isnull(m_open1)) m_open1 = 0;
        if (wo_isnull(i1)) i1 = 0;
        if (wo_isnull(d1)) d1 = 0;
        if (wo_isnull(m_open2)) m_open2 = 0;
        if (wo_isnull(i2)) i2 = 0;
        if (wo_isnull(d2)) d2 = 0;
        if (!m_misms && !m_open1 && !i1 && !d1 && !m_open2 && !i2 && !d2) {
            ++num_null;
            continue;
        }
        num_null = 0;
        /* limits: a null input contributes the null wavefront's lo=1, hi=-1 */
#define LO(w) ((w) ? (w)->lo : 1)
#define HI(w) ((w) ? (w)->hi : -1)
        int lo = LO(m_misms), hi = HI(m_misms);
        if (lo > LO(m_open1) - 1) lo = LO(m_open1) - 1;
        if (hi < HI(m_open1) + 1) hi = HI(m_open1) + 1;
        if (lo > LO(i1) + 1) lo = LO(i1) + 1;
        if (hi < HI(i1) + 1) hi = HI(i1) + 1;
        if (lo > LO(d1) - 1) lo = LO(d1) - 1;
        if (hi < HI(d1) - 1) hi = HI(d1) - 1;
        if (lo > LO(m_open2) - 1) lo = LO(m_open2) - 1;
        if (hi < HI(m_open2) + 1) hi = HI(m_open2) + 1;
        if (lo > LO(i2) + 1) lo = LO(i2) + 1;
        if (hi < HI(i2) + 1) hi = HI(i2) + 1;
        if (lo > LO(d2) - 1) lo = LO(d2) - 1;
        if (hi < HI(d2) - 1) hi = HI(d2) - 1;
#undef LO
#undef HI
        wo_wf *oM = wo_new(lo, hi);
        wo_wf *oI1 = (m_open1 || i1) ? wo_new(lo, hi) : 0;
        wo_wf *oD1 = (m_open1 || d1) ? wo_new(lo, hi) : 0;
        wo_wf *oI2 = (m_open2 || i2) ? wo_new(lo, hi) : 0;
        wo_wf *oD2 = (m_open2 || d2) ? wo_new(lo, hi) : 0;
        for (int k = lo; k <= hi; ++k) {
            const int32_t ins1 = mx(wo_get(m_open1, k - 1), wo_get(i1, k - 1)) + 1;
            const int32_t ins2 = mx(wo_get(m_open2, k - 1), wo_get(i2, k - 1)) + 1;
            const int32_t del1 = mx(wo_get(m_open1, k + 1), wo_get(d1, k + 1));
            const int32_t del2 = mx(wo_get(m_open2, k + 1), wo_get(d2, k + 1));
            const int32_t misms = wo_get(m_misms, k) + 1;
            int32_t best = mx(mx(del1, del2), mx(misms, mx(ins1, ins2)));
            const uint32_t h = (uint32_t)best, v = (uint32_t)(best - k);
            if (h > (uint32_t)tlen || v > (uint32_t)plen) best = WO_NULL;
            oM->off[k - lo] = best;
            if (oI1) oI1->off[k - lo] = ins1;
            if (oI2) oI2->off[k - lo] = ins2;
            if (oD1) oD1->off[k - lo] = del1;
            if (oD2) oD2->off[k - lo] = del2;
        }
        wo_trim(oM, plen, tlen);
        if (oI1) wo_trim(oI1, plen, tlen);
        if (oD1) wo_trim(oD1, plen, tlen);
        if (oI2) wo_trim(oI2, plen, tlen);
        if (oD2) wo_trim(oD2, plen, tlen);
        W[s].M = oM, W[s].I1 = oI1, W[s].D1 = oD1, W[s].I2 = oI2, W[s].D2 = oD2;
    }
    /* backtrace into a reversed buffer */
    const int maxops = 2 * (plen + tlen) + 8;
    char *rev = (char *)malloc((size_t)maxops);
    int n = 0;
    if (status == 0) {
        const int plen_ = plen, tlen_ = tlen;
        if (!singletrack) {
            /* wavefront_backtrace_affine: piggyback (offset<<4 | type), M=9 > D2ext=8 > ... > I1open=1 */
            enum { BM = 9, BD2E = 8, BD2O = 7, BD1E = 6, BD1O = 5, BI2E = 4, BI2O = 3, BI1E = 2, BI1O = 1 };
            int mt = 0; /* 0 M, 1 I1, 2 I2, 3 D1, 4 D2 */
            int sc = end_score, k = k_end;
            int32_t off = tlen;
            int h = off, v = off - k;
#define PB(o, t) ((int64_t)((((uint64_t)(int64_t)(o)) << 4) | (uint64_t)(t)))
#define SG(arr, scr) ((scr) >= 0 ? W[(scr)].arr : 0)
            while (v > 0 && h > 0 && sc > 0) {
                const int smm = sc - x, sg1 = sc - o1 - e1, sg2 = sc - o2 - e2, sx1 = sc - e1, sx2 = sc - e2;
                int64_t mall;
                const int64_t misms = smm >= 0 && SG(M, smm) ? PB(wo_get(SG(M, smm), k) + 1, BM) : PB(WO_NULL, 0);
                const int64_t i1o = sg1 >= 0 && SG(M, sg1) ? PB(wo_get(SG(M, sg1), k - 1) + 1, BI1O) : PB(WO_NULL, 0);
                const int64_t i1e = sx1 >= 0 && SG(I1, sx1) ? PB(wo_get(SG(I1, sx1), k - 1) + 1, BI1E) : PB(WO_NULL, 0);
                const int64_t d1o = sg1 >= 0 && SG(M, sg1) ? PB(wo_get(SG(M, sg1), k + 1), BD1O) : PB(WO_NULL, 0);
                const int64_t d1e = sx1 >= 0 && SG(D1, sx1) ? PB(wo_get(SG(D1, sx1), k + 1), BD1E) : PB(WO_NULL, 0);
                const int64_t i2o = sg2 >= 0 && SG(M, sg2) ? PB(wo_get(SG(M, sg2), k - 1) + 1, BI2O) : PB(WO_NULL, 0);
                const int64_t i2e = sx2 >= 0 && SG(I2, sx2) ? PB(wo_get(SG(I2, sx2), k - 1) + 1, BI2E) : PB(WO_NULL, 0);
                const int64_t d2o = sg2 >= 0 && SG(M, sg2) ? PB(wo_get(SG(M, sg2), k + 1), BD2O) : PB(WO_NULL, 0);
                const int64_t d2e = sx2 >= 0 && SG(D2, sx2) ? PB(wo_get(SG(D2, sx2), k + 1), BD2E) : PB(WO_NULL, 0);
#define MX64(a, b) ((a) > (b) ? (a) : (b))
                switch (mt) {
                case 0: mall = MX64(misms, MX64(MX64(MX64(i1o, i1e), MX64(i2o, i2e)), MX64(MX64(d1o, d1e), MX64(d2o, d2e)))); break;
                case 1: mall = MX64(i1o, i1e); break;
                case 2: mall = MX64(i2o, i2e); break;
                case 3: mall = MX64(d1o, d1e); break;
                default: mall = MX64(d2o, d2e); break;
                }
                if (mall < 0) break;
                if (mt == 0) {
                    const int mo = (int)(mall >> 4);
                    for (int i = 0; i < off - mo; ++i) rev[n++] = 'M';
                    off = mo;
                    v = off - k, h = off;
                    if (v <= 0 || h <= 0) break;
                }
                const int bt = (int)(mall & 0xf);
                switch (bt) {
                case BM: sc = smm; mt = 0; break;
                case BI1O: sc = sg1; mt = 0; break;
                case BI1E: sc = sx1; mt = 1; break;
                case BI2O: sc = sg2; mt = 0; break;
                case BI2E: sc = sx2; mt = 2; break;
                case BD1O: sc = sg1; mt = 0; break;
                case BD1E: sc = sx1; mt = 3; break;
                case BD2O: sc = sg2; mt = 0; break;
                default: sc = sx2; mt = 4; break;
                }
                if (bt == BM) rev[n++] = 'X', --off;
                else if (bt <= BI2E) rev[n++] = 'I', --k, --off;
                else rev[n++] = 'D', ++k;
                v = off - k, h = off;
            }
            if (mt == 0) {
                if (v > 0 && h > 0) {
                    const int nm = v < h ? v : h;
                    for (int i = 0; i < nm; ++i) rev[n++] = 'M';
                    v -= nm, h -= nm;
                }
                while (v > 0) rev[n++] = 'D', --v;
                while (h > 0) rev[n++] = 'I', --h;
            }
#undef MX64
#undef SG
#undef PB
        } else {
            /* wavefront_backtrace_affine_singletrack: only M wavefronts are consulted */
            int sc = end_score, k = k_end, in_m = 1, gl = 0;
            int32_t off = tlen, off_be = off;
            const int64_t maxgap = (int64_t)plen_ + tlen_;
            int ok = 1;
            while (sc != 0) {
                if (sc < 0 || off < 0) { ok = 0; break; }
                if (in_m) {
                    const int v = off - k, h = off;
                    if (v < 0 || h < 0 || v > plen_ || h > tlen_) { ok = 0; break; }
                    int nm = 0;
                    while (nm < v && nm < h && pattern[v - nm - 1] == text[h - nm - 1]) ++nm;
                    off_be = off - nm;
                    const int ms = sc - x;
                    const wo_wf *mw = ms >= 0 ? W[ms].M : 0;
                    if (mw && mw->lo <= k && k <= mw->hi && mw->off[k - mw->base] + 1 == off_be) {
                        for (int i = 0; i < nm; ++i) rev[n++] = 'M';
                        rev[n++] = 'X';
                        off = off_be - 1;
                        sc = ms;
                    } else {
                        in_m = 0, gl = 0;
                    }
                    continue;
                }
                ++gl;
                if ((int64_t)gl > maxgap) { ok = 0; break; }
                const int ki = k - gl, kd = k + gl;
                int done = 0;
                for (int piece = 0; piece < 2 && !done; ++piece) {
                    const int64_t isc = piece == 0 ? (int64_t)sc - o1 - (int64_t)gl * e1 : (int64_t)sc - o2 - (int64_t)gl * e2;
                    const wo_wf *iw = (isc >= 0 && isc < cap) ? W[isc].M : 0;
                    if (iw && iw->lo <= ki && ki <= iw->hi && iw->off[ki - iw->base] + gl >= off_be &&
                        iw->off[ki - iw->base] + gl <= off) {
                        const int nm = off - (iw->off[ki - iw->base] + gl);
                        for (int i = 0; i < nm; ++i) rev[n++] = 'M';
                        for (int i = 0; i < gl; ++i) rev[n++] = 'I';
                        k = ki, off = iw->off[ki - iw->base], sc = (int)isc, in_m = 1, done = 1;
                    } else if (iw && iw->lo <= kd && kd <= iw->hi && iw->off[kd - iw->base] >= off_be &&
                               iw->off[kd - iw->base] <= off) {
                        const int nm = off - iw->off[kd - iw->base];
                        for (int i = 0; i < nm; ++i) rev[n++] = 'M';
                        for (int i = 0; i < gl; ++i) rev[n++] = 'D';
                        k = kd, off = iw->off[kd - iw->base], sc = (int)isc, in_m = 1, done = 1;
                    }
                }
            }
            if (ok && (!in_m || k != 0 || off < 0 || off > plen_ || off > tlen_)) ok = 0;
            if (ok)
                for (int i = 0; i < off; ++i)
                    if (pattern[i] != text[i]) { ok = 0; break; }
            if (ok)
                for (int i = 0; i < off; ++i) rev[n++] = 'M';
            if (!ok) status = -300;
        }
    }
    if (status == 0) {
        *score_out = -end_score;
        *n_ops = n;
        if (ops && n <= ops_cap)
            for (int i = 0; i < n; ++i) ops[i] = rev[n - 1 - i];
    }
    free(rev);
    for (int i = 0; i <= s && i < cap; ++i) {
        wo_free(W[i].M), wo_free(W[i].I1), wo_free(W[i].D1), wo_free(W[i].I2), wo_free(W[i].D2);
    }
    free(W);
    return status;
}
