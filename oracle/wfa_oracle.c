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
 *   medium / low memory       (memory_mode 1 / 2, wavefront/wavefront_attributes.h:122-127)
 *     piggyback kernel        wavefront/wavefront_compute_affine2p.c:110-282
 *                             (the gap-affine delegate :291-299 has the same ties)
 *     occupancy + offload     wavefront/wavefront_backtrace_offload.c:39-71, :130-288
 *     BT-buffer               wavefront/wavefront_backtrace_buffer.c:219-247
 *     pcigar traceback        wavefront/wavefront_backtrace.c:767-799,
 *                             wavefront/wavefront_backtrace_buffer.c:251-265, :323-366,
 *                             wavefront/wavefront_pcigar.c:222-278
 *   (Singletrack is only honoured in high memory, wavefront/wavefront_aligner.c:251-260.)
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
    uint32_t *pc;    /* piggyback: packed CIGAR of the cell's last operations */
    uint32_t *pv;    /* piggyback: BT-block holding the operations before them */
    int occ;         /* piggyback: bt_occupancy_max */
} wo_wf;

/* Packed CIGAR (wavefront/wavefront_pcigar.h:44-71): 2 bits per operation, newest in the
 * low bits: 1 deletion, 2 mismatch (or gap close), 3 insertion; 16 operations per word. */
#define WO_PC_FULL 0x40000000u
#define WO_PC_ALMOST_FULL 0x10000000u /* 15 operations or more */
#define WO_PC_HALF_FULL 0x00010000u   /* 9 operations or more */
#define WO_BT_NULL 0xFFFFFFFFu

typedef struct {
    uint32_t pc, prev;
} wo_blk;
typedef struct {
    wo_blk *b;
    size_t n, cap;
} wo_blocks;
static uint32_t wo_blk_push(wo_blocks *B, uint32_t pc, uint32_t prev) {
    if (B->n == B->cap) {
        B->cap = B->cap ? 2 * B->cap : 1024;
        B->b = (wo_blk *)realloc(B->b, sizeof(wo_blk) * B->cap);
    }
    B->b[B->n].pc = pc, B->b[B->n].prev = prev;
    return (uint32_t)B->n++;
}

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
static __thread int wo_bt = 0; /* the aligner runs in a piggyback memory mode */
static wo_wf *wo_new(int lo, int hi) {
    wo_wf *w = (wo_wf *)malloc(sizeof(wo_wf));
    const size_t len = (size_t)(hi - lo + 1 > 0 ? hi - lo + 1 : 1);
    wo_ints_allocated += (long long)len;
    w->lo = lo, w->hi = hi, w->base = lo;
    w->off = (int32_t *)malloc(sizeof(int32_t) * len);
    w->pc = wo_bt ? (uint32_t *)calloc(len, sizeof(uint32_t)) : 0;
    w->pv = wo_bt ? (uint32_t *)malloc(sizeof(uint32_t) * len) : 0;
    w->occ = 0;
    return w;
}
static void wo_free(wo_wf *w) {
    if (w) free(w->off), free(w->pc), free(w->pv), free(w);
}
static uint32_t wo_getpc(const wo_wf *w, int k) {
    if (!w || w->lo > w->hi || k < w->lo || k > w->hi) return 0;
    return w->pc[k - w->base];
}
static uint32_t wo_getpv(const wo_wf *w, int k) {
    if (!w || w->lo > w->hi || k < w->lo || k > w->hi) return WO_BT_NULL;
    return w->pv[k - w->base];
}
/* wavefront_backtrace_offload_blocks_selective: every cell of [lo, hi] with an offset and
 * at least the mask's operations moves its packed CIGAR into a new BT-block. */
static void wo_offload(wo_wf *w, int lo, int hi, uint32_t mask, wo_blocks *B) {
    for (int k = lo; k <= hi; ++k) {
        if (w->off[k - w->base] >= 0 && w->pc[k - w->base] >= mask) {
            const uint32_t idx = wo_blk_push(B, w->pc[k - w->base], w->pv[k - w->base]);
            w->pc[k - w->base] = 0;
            w->pv[k - w->base] = idx;
        }
    }
}
static int wo_lcp(const char *pattern, int plen, const char *text, int tlen, int v, int h) {
    int n = 0;
    while (v + n < plen && h + n < tlen && pattern[v + n] == text[h + n]) ++n;
    return n;
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
int oracle_wfa_align_mode(const char *pattern, int plen, const char *text, int tlen, int x, int o1, int e1,
                          int o2, int e2, int singletrack, int memory_mode, int *score_out, char *ops, int ops_cap,
                          int *n_ops) {
    *score_out = 0, *n_ops = 0;
    wo_ints_allocated = 0;
    const int bt = memory_mode == 1 || memory_mode == 2;
    if (bt) singletrack = 0;
    wo_bt = bt;
    wo_blocks B = {0, 0, 0};
    const int scope = (o1 + e1 > o2 + e2 ? o1 + e1 : o2 + e2);
    const int max_score_scope = (scope > x ? scope : x) + 1;
    int cap = 1024, s = 0, num_null = 0;
    wo_score *W = (wo_score *)calloc((size_t)cap, sizeof(wo_score));
    W[0].M = wo_new(0, 0);
    W[0].M->off[0] = 0;
    if (bt) { /* initial BT-block: start position (0, 0), no predecessor */
        W[0].M->pc[0] = 0;
        W[0].M->pv[0] = wo_blk_push(&B, 0, WO_BT_NULL);
    }
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
            if (bt) {
                /* each gap cell takes the extension on a tie; M prefers the mismatch, then
                 * D2, D1, I2, I1 (the last equal candidate assigned wins) */
                uint32_t i1pc, i1pv, i2pc, i2pv, d1pc, d1pv, d2pc, d2pv, mpc = 0, mpv = WO_BT_NULL;
                if (wo_get(i1, k - 1) >= wo_get(m_open1, k - 1)) i1pc = wo_getpc(i1, k - 1), i1pv = wo_getpv(i1, k - 1);
                else i1pc = wo_getpc(m_open1, k - 1), i1pv = wo_getpv(m_open1, k - 1);
                if (wo_get(i2, k - 1) >= wo_get(m_open2, k - 1)) i2pc = wo_getpc(i2, k - 1), i2pv = wo_getpv(i2, k - 1);
                else i2pc = wo_getpc(m_open2, k - 1), i2pv = wo_getpv(m_open2, k - 1);
                if (wo_get(d1, k + 1) >= wo_get(m_open1, k + 1)) d1pc = wo_getpc(d1, k + 1), d1pv = wo_getpv(d1, k + 1);
                else d1pc = wo_getpc(m_open1, k + 1), d1pv = wo_getpv(m_open1, k + 1);
                if (wo_get(d2, k + 1) >= wo_get(m_open2, k + 1)) d2pc = wo_getpc(d2, k + 1), d2pv = wo_getpv(d2, k + 1);
                else d2pc = wo_getpc(m_open2, k + 1), d2pv = wo_getpv(m_open2, k + 1);
                i1pc = (i1pc << 2) | 3u, i2pc = (i2pc << 2) | 3u;
                d1pc = (d1pc << 2) | 1u, d2pc = (d2pc << 2) | 1u;
                const int32_t mmax = mx(mx(del1, del2), mx(misms, mx(ins1, ins2)));
                if (mmax == ins1) mpc = i1pc, mpv = i1pv;
                if (mmax == ins2) mpc = i2pc, mpv = i2pv;
                if (mmax == del1) mpc = d1pc, mpv = d1pv;
                if (mmax == del2) mpc = d2pc, mpv = d2pv;
                if (mmax == misms) mpc = wo_getpc(m_misms, k), mpv = wo_getpv(m_misms, k);
                oM->pc[k - lo] = (mpc << 2) | 2u, oM->pv[k - lo] = mpv;
                if (oI1) oI1->pc[k - lo] = i1pc, oI1->pv[k - lo] = i1pv;
                if (oI2) oI2->pc[k - lo] = i2pc, oI2->pv[k - lo] = i2pv;
                if (oD1) oD1->pc[k - lo] = d1pc, oD1->pv[k - lo] = d1pv;
                if (oD2) oD2->pc[k - lo] = d2pc, oD2->pv[k - lo] = d2pv;
            }
        }
        if (bt) {
            /* occupancy bound of every output (wavefront_backtrace_offload_occupation_affine) */
            int occ_i1 = 0, occ_d1 = 0, occ_i2 = 0, occ_d2 = 0, occ_m = 0;
            if (m_open1) occ_i1 = occ_d1 = m_open1->occ + 1;
            if (i1 && occ_i1 < i1->occ + 1) occ_i1 = i1->occ + 1;
            if (d1 && occ_d1 < d1->occ + 1) occ_d1 = d1->occ + 1;
            if (m_open2) occ_i2 = occ_d2 = m_open2->occ + 1;
            if (i2 && occ_i2 < i2->occ + 1) occ_i2 = i2->occ + 1;
            if (d2 && occ_d2 < d2->occ + 1) occ_d2 = d2->occ + 1;
            if (m_misms) occ_m = m_misms->occ;
            if (occ_m < occ_i1) occ_m = occ_i1;
            if (occ_m < occ_i2) occ_m = occ_i2;
            if (occ_m < occ_d1) occ_m = occ_d1;
            if (occ_m < occ_d2) occ_m = occ_d2;
            ++occ_m;
            oM->occ = occ_m;
            if (oI1) oI1->occ = occ_i1;
            if (oD1) oD1->occ = occ_d1;
            if (oI2) oI2->occ = occ_i2;
            if (oD2) oD2->occ = occ_d2;
            /* offload the outputs that may fill up: medium moves half-full words and
             * resumes at 8, low moves words of 15 or more and resumes at 14 */
            const uint32_t mask = memory_mode == 1 ? WO_PC_HALF_FULL : WO_PC_ALMOST_FULL;
            const int resume = memory_mode == 1 ? 8 : 14;
            wo_wf *outs[5] = {oM, oI1, oD1, oI2, oD2};
            for (int c = 0; c < 5; ++c) {
                if (outs[c] && outs[c]->occ >= 15) {
                    wo_offload(outs[c], lo, hi, mask, &B);
                    outs[c]->occ = resume;
                }
            }
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
    int fwd = 0; /* the piggyback traceback writes the operations in order */
    if (status == 0 && bt) {
        /* wavefront_backtrace_pcigar: collect the packed CIGARs from the end cell back to
         * the initial block, then unpack them oldest first, extending the matches before
         * every operation taken in M and dropping the mismatch that closes a gap */
        const wo_wf *mw = W[end_score].M;
        uint32_t cur_pc = mw->pc[k_end - mw->base], cur_prev = mw->pv[k_end - mw->base];
        size_t nb = 0, cb = 64;
        uint32_t *chain = (uint32_t *)malloc(sizeof(uint32_t) * cb);
        while (cur_prev != WO_BT_NULL) {
            if (nb == cb) cb *= 2, chain = (uint32_t *)realloc(chain, sizeof(uint32_t) * cb);
            chain[nb++] = cur_pc;
            cur_pc = B.b[cur_prev].pc, cur_prev = B.b[cur_prev].prev;
        }
        /* cur_pc is now the initial block's start-position record: (0, 0) end to end */
        int v = 0, h = 0, in_m = 1;
        for (size_t i = nb; i-- > 0;) {
            uint32_t pc = chain[i];
            int len = 16;
            if (pc < WO_PC_FULL) {
                const int free_slots = pc ? __builtin_clz(pc) / 2 : 16;
                len -= free_slots;
                if (len > 0) pc <<= free_slots * 2;
            }
            for (int j = 0; j < len; ++j) {
                if (in_m) {
                    const int nm = wo_lcp(pattern, plen, text, tlen, v, h);
                    for (int t = 0; t < nm; ++t) rev[n++] = 'M';
                    v += nm, h += nm;
                }
                const uint32_t op = pc >> 30;
                pc <<= 2;
                if (!in_m && op == 2u) {
                    in_m = 1;
                    continue;
                }
                rev[n++] = op == 1u ? 'D' : op == 2u ? 'X' : op == 3u ? 'I' : '?';
                v += op == 1u || op == 2u;
                h += op == 2u || op == 3u;
                in_m = op == 2u;
            }
        }
        free(chain);
        const int nm = (plen - v) < (tlen - h) ? (plen - v) : (tlen - h);
        for (int t = 0; t < nm; ++t) rev[n++] = 'M';
        v += nm, h += nm;
        while (h < tlen) rev[n++] = 'I', ++h;
        while (v < plen) rev[n++] = 'D', ++v;
        fwd = 1;
    } else if (status == 0) {
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
            for (int i = 0; i < n; ++i) ops[i] = fwd ? rev[i] : rev[n - 1 - i];
    }
    free(rev);
    free(B.b);
    wo_bt = 0;
    for (int i = 0; i <= s && i < cap; ++i) {
        wo_free(W[i].M), wo_free(W[i].I1), wo_free(W[i].D1), wo_free(W[i].I2), wo_free(W[i].D2);
    }
    free(W);
    return status;
}

int oracle_wfa_align(const char *pattern, int plen, const char *text, int tlen, int x, int o1, int e1, int o2, int e2,
                     int singletrack, int *score_out, char *ops, int ops_cap, int *n_ops) {
    return oracle_wfa_align_mode(pattern, plen, text, tlen, x, o1, e1, o2, e2, singletrack, 0, score_out, ops, ops_cap,
                                 n_ops);
}
