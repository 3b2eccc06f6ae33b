/*
 * ksw2_oracle.c -- TEST INFRASTRUCTURE (oracle).  A plain-C, scalar
 * restatement of AnchorWave's KSW2 extd2 two-piece-affine DP, written to be
 * byte-for-byte equivalent to the reference SIMD kernels so it can check the
 * CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg use it; nothing in the product path links it.
 *
 * Parity pin: tests/test_oracle.py compares every ksw_extz_t field and the
 * CIGAR of this restatement against the compiled reference
 * (oracle/_ref/libawref_<isa>.so) over seeded corpora and edge cases.
 *
 * What is restated (reference file:line):
 *   ksw_extd2_avx512          minimap2/ksw2_extd2_avx.c:51-787  (block = 64)
 *   ksw_extd2_avx2            minimap2/ksw2_extd2_avx.c:800-1575 (block = 32)
 *   ksw_extd2_sse             minimap2/ksw2_extd2_sse.c:39-419   (block = 16)
 *   ksw_backtrack             minimap2/ksw2.h:160-192
 *   ksw_push_cigar            minimap2/ksw2.h:144-154
 *   ksw_reset_extz            minimap2/ksw2.h:194-199
 *   ksw_apply_zdrop           minimap2/ksw2.h:201-217
 *   ksw2_singletrack_backtrace_affine2p  minimap2/ksw2_singletrack.cpp:63-176
 *   ksw_extd2_singletrack_sse  minimap2/ksw2_singletrack.cpp:202-626 (block = 16 with the
 *                              Singletrack flag: the same DP and tracks, minimap2's original
 *                              end rules -- mqe/mte on a strict ">", mte_q = r - en with en
 *                              rounded up to its 16-byte block, :583-586 -- and the
 *                              reconstruction whatever the EXTZ/SEMIGLOBAL flags, :606-615)
 *
 * The SIMD kernels keep difference-encoded int8 cells (u,v,x,y,x2,y2) in
 * arrays indexed by target position t, and recompute every anti-diagonal r
 * over whole SIMD blocks.  Cells outside the band but inside the block
 * rounding ("padding lanes") are computed from whatever the arrays held, and
 * in banded mode the in-band cells and the traceback DO read them, so this
 * restatement keeps the same arrays, the same memory layout behind the score
 * fill, and the same per-block lane rules.  All int8 arithmetic wraps.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

#define OR_NEG_INF (-0x40000000)

#define OR_SCORE_ONLY     0x01
#define OR_RIGHT          0x02
#define OR_GENERIC_SC     0x04
#define OR_APPROX_MAX     0x08
#define OR_APPROX_DROP    0x10
#define OR_EXTZ_ONLY      0x40
#define OR_REV_CIGAR      0x80
#define OR_SEMIGLOBAL_END 0x800
#define OR_SINGLETRACK    0x1000

/* Same layout as ksw_extz_t (minimap2/ksw2.h:40-50). */
typedef struct {
    uint32_t max:31, zdropped:1;
    int max_q, max_t;
    int mqe, mqe_t;
    int mte, mte_q;
    int score;
    int m_cigar, n_cigar;
    int reach_end;
    int stopped;
    uint32_t *cigar;
} or_extz_t;

static inline int8_t w8(int v) { return (int8_t)(uint8_t)(v & 0xff); }
static inline int8_t max8(int8_t a, int8_t b) { return a > b ? a : b; }
static inline int8_t min8(int8_t a, int8_t b) { return a < b ? a : b; }

/* minimap2/ksw2.h:194-199 */
static void or_reset(or_extz_t *ez) {
    ez->max_q = ez->max_t = ez->mqe_t = ez->mte_q = -1;
    ez->max = 0, ez->score = ez->mqe = ez->mte = OR_NEG_INF;
    ez->n_cigar = 0, ez->zdropped = 0, ez->reach_end = 0, ez->stopped = 0;
}

/* minimap2/ksw2.h:144-154: BAM op (len<<4 | op), merged with the last op. */
static uint32_t *or_push(int *n, int *m, uint32_t *c, uint32_t op, int len) {
    if (*n == 0 || op != (c[*n - 1] & 0xf)) {
        if (*n == *m) {
            *m = *m ? (*m) << 1 : 4;
            c = (uint32_t *)realloc(c, (size_t)(*m) << 2);
        }
        c[(*n)++] = (uint32_t)len << 4 | op;
    } else
        c[*n - 1] += (uint32_t)len << 4;
    return c;
}

/* minimap2/ksw2.h:201-217 with is_rot = 1 (a = r, b = t). */
static int or_zdrop(or_extz_t *ez, int32_t H, int r, int t, int zdrop, int8_t e) {
    if (H > (int32_t)ez->max) {
        ez->max = (uint32_t)H, ez->max_t = t, ez->max_q = r - t;
    } else if (t >= ez->max_t && r - t >= ez->max_q) {
        int tl = t - ez->max_t, ql = (r - t) - ez->max_q;
        int l = tl > ql ? tl - ql : ql - tl;
        if (zdrop >= 0 && (int)ez->max - H > zdrop + l * e) {
            ez->zdropped = 1;
            return 1;
        }
    }
    return 0;
}

/* minimap2/ksw2.h:160-192, anti-diagonal ("rotated") layout, no introns. */
static void or_backtrack(int is_rev, const uint8_t *p, const int *off, const int *off_end,
                         size_t n_col, int i0, int j0, int *m_cigar_, int *n_cigar_,
                         uint32_t **cigar_) {
    int n_cigar = 0, m_cigar = *m_cigar_, i = i0, j = j0, state = 0;
    uint32_t *cigar = *cigar_;
    while (i >= 0 && j >= 0) {
        int r = i + j, force = -1;
        uint32_t cell;
        if (i < off[r]) force = 2;
        if (off_end && i > off_end[r]) force = 1;
        cell = force < 0 ? p[(size_t)r * n_col + (size_t)(i - off[r])] : 0;
        if (state == 0) state = cell & 7;
        else if (!(cell >> (state + 2) & 1)) state = 0;
        if (state == 0) state = cell & 7;
        if (force >= 0) state = force;
        if (state == 0) cigar = or_push(&n_cigar, &m_cigar, cigar, 0, 1), --i, --j;
        else if (state == 1 || state == 3) cigar = or_push(&n_cigar, &m_cigar, cigar, 2, 1), --i;
        else cigar = or_push(&n_cigar, &m_cigar, cigar, 1, 1), --j;
    }
    if (i >= 0) cigar = or_push(&n_cigar, &m_cigar, cigar, 2, i + 1);
    if (j >= 0) cigar = or_push(&n_cigar, &m_cigar, cigar, 1, j + 1);
    if (!is_rev)
        for (i = 0; i < n_cigar >> 1; ++i) {
            uint32_t tmp = cigar[i];
            cigar[i] = cigar[n_cigar - 1 - i], cigar[n_cigar - 1 - i] = tmp;
        }
    *m_cigar_ = m_cigar, *n_cigar_ = n_cigar, *cigar_ = cigar;
}

/* ---- Singletrack reconstruction, minimap2/ksw2_singletrack.cpp:23-176 ---- */

static int32_t st_gap(int32_t l, int32_t o1, int32_t e1, int32_t o2, int32_t e2) {
    if (l <= 0) return 0;
    int64_t a = (int64_t)o1 + (int64_t)l * e1, b = (int64_t)o2 + (int64_t)l * e2;
    return (int32_t)(a > b ? a : b);
}

static int32_t st_diff(const int8_t *mtx, int32_t i, int32_t j, size_t n_col, const int *off,
                       const int *off_end, int32_t o1, int32_t e1, int32_t o2, int32_t e2) {
    if (i < 0 || j < 0) {
        int32_t c = i < 0 ? j : i;
        return st_gap(c + 1, o1, e1, o2, e2) - st_gap(c, o1, e1, o2, e2);
    }
    int64_t d = (int64_t)i + j;
    if (i < off[d] || i > off_end[d]) return OR_NEG_INF;
    return (int32_t)mtx[(size_t)d * n_col + (size_t)(i - off[d])];
}

static int st_finite(int32_t v) { return v > OR_NEG_INF / 2 && v < -OR_NEG_INF / 2; }

static void or_singletrack_bt(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                              int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2,
                              int8_t e2, size_t n_col, const int *off, const int *off_end,
                              const int8_t *p, const int8_t *p2, or_extz_t *ez) {
    const int32_t o1 = -q, g1 = -e, o2 = -q2, g2 = -e2;
    int in_m = 1, n_cigar = 0, m_cigar = ez->m_cigar, valid = 1;
    uint32_t *cigar = ez->cigar;
    int32_t i = tlen - 1, j = qlen - 1, l = 0, dd = 0, di = 0;
    while (i >= 0 && j >= 0) {
        int32_t dg = i + j;
        if (i < off[dg]) { cigar = or_push(&n_cigar, &m_cigar, cigar, 1, 1); --j; in_m = 1; continue; }
        if (i > off_end[dg]) { cigar = or_push(&n_cigar, &m_cigar, cigar, 2, 1); --i; in_m = 1; continue; }
        if (in_m) {
            int32_t h = st_diff(p, i, j, n_col, off, off_end, o1, g1, o2, g2);
            int32_t v = st_diff(p2, i, j - 1, n_col, off, off_end, o1, g1, o2, g2);
            int32_t cost = mat[target[i] * m + query[j]];
            if (st_finite(h) && st_finite(v) && (int64_t)h + v == cost) {
                cigar = or_push(&n_cigar, &m_cigar, cigar, 0, 1);
                --i, --j;
            } else {
                in_m = 0, l = 0;
                di = st_diff(p, i, j, n_col, off, off_end, o1, g1, o2, g2);
                dd = st_diff(p2, i, j, n_col, off, off_end, o1, g1, o2, g2);
            }
        } else {
            ++l;
            if (l > i + 1 && l > j + 1) { valid = 0; break; }
            int32_t a1 = o1 + l * g1, a2 = o2 + l * g2, jn = j - l, id = i - l;
            if (id >= -1 && (dd == a1 || dd == a2)) {
                cigar = or_push(&n_cigar, &m_cigar, cigar, 2, l);
                i = id, in_m = 1;
            } else if (jn >= -1 && (di == a1 || di == a2)) {
                cigar = or_push(&n_cigar, &m_cigar, cigar, 1, l);
                j = jn, in_m = 1;
            } else {
                if (jn >= 0) {
                    int32_t H = st_diff(p, i, jn, n_col, off, off_end, o1, g1, o2, g2);
                    di = (st_finite(di) && st_finite(H)) ? di + H : OR_NEG_INF;
                }
                if (id >= 0) {
                    int32_t V = st_diff(p2, id, j, n_col, off, off_end, o1, g1, o2, g2);
                    dd = (st_finite(dd) && st_finite(V)) ? dd + V : OR_NEG_INF;
                }
            }
        }
    }
    if (!valid) {
        free(cigar);
        ez->cigar = 0, ez->m_cigar = ez->n_cigar = 0;
        return;
    }
    if (i >= 0) cigar = or_push(&n_cigar, &m_cigar, cigar, 2, i + 1);
    if (j >= 0) cigar = or_push(&n_cigar, &m_cigar, cigar, 1, j + 1);
    for (i = 0; i < n_cigar >> 1; ++i) {
        uint32_t tmp = cigar[i];
        cigar[i] = cigar[n_cigar - 1 - i], cigar[n_cigar - 1 - i] = tmp;
    }
    ez->cigar = cigar, ez->m_cigar = m_cigar, ez->n_cigar = n_cigar;
}

/* ---- the DP ------------------------------------------------------------- */

/*
 * block: SIMD width in bytes of the reference kernel restated (64 = AVX-512,
 * 32 = AVX2, 16 = SSE).  stop_interval/stop_at emulate the cooperative
 * progress hook of minimap2/ksw2_progress.c:30-38 (stop_at < 0 disables):
 * anti-diagonal r is abandoned when r % stop_interval == 0 && r >= stop_at.
 */
void oracle_ksw_extd2(int block, int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                      int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                      int w, int zdrop, int end_bonus, int flag, int stop_interval, int stop_at,
                      or_extz_t *ez) {
    const int B = block;
    /* qe is taken BEFORE the q+e <= q2+e2 swap (it is initialised at its
     * declaration in ksw2_extd2_sse.c:73 / ksw2_extd2_avx.c:113); it only seeds
     * H[0] and the approximate-max H0, so every H shifts when the swap fires. */
    int r, t, qe = q + e, n_col_, *off = 0, *off_end = 0, tlen_, qlen_, last_st, last_en;
    int max_sc, min_sc, long_thres, long_diff, wl, wr;
    int with_cigar = !(flag & OR_SCORE_ONLY), approx_max = !!(flag & OR_APPROX_MAX);
    int singletrack = !!(flag & OR_SINGLETRACK);
    const int sse_st = singletrack && B == 16; /* ksw_extd2_singletrack_sse */
    int32_t *H = 0, H0 = 0, last_H0_t = 0;
    int8_t *mem, *u, *v, *x, *y, *x2, *y2, *s;
    uint8_t *sf, *qr, *p = 0, *p2 = 0;
    int8_t sc_mch, sc_mis, sc_N, m1;
    size_t T, n_diag, row;

    or_reset(ez);
    if (m <= 1 || qlen <= 0 || tlen <= 0) return;
    if (B > 16 && qlen > INT_MAX - tlen + 1) { ez->zdropped = 1; return; }
    /* ksw2_extd2_sse.c:83 -- make q+e no larger than q2+e2 */
    if (q2 + e2 < q + e) { int8_t tq = q, te = e; q = q2, e = e2, q2 = tq, e2 = te; }
    sc_mch = mat[0], sc_mis = mat[1];
    sc_N = mat[m * m - 1] == 0 ? w8(-e2) : mat[m * m - 1];
    m1 = (int8_t)(m - 1);

    if (w < 0) w = tlen > qlen ? tlen : qlen;
    wl = wr = w;
    tlen_ = (tlen + B - 1) / B;
    n_col_ = qlen < tlen ? qlen : tlen;
    n_col_ = ((n_col_ < w + 1 ? n_col_ : w + 1) + B - 1) / B + 1;
    qlen_ = (qlen + B - 1) / B;
    for (t = 1, max_sc = mat[0], min_sc = mat[1]; t < m * m; ++t) {
        max_sc = max_sc > mat[t] ? max_sc : mat[t];
        min_sc = min_sc < mat[t] ? min_sc : mat[t];
    }
    (void)max_sc;
    if (-min_sc > 2 * (q + e)) return;

    /* ksw2_extd2_sse.c:107-110 -- where the long-gap piece takes over */
    long_thres = e != e2 ? (q2 - q) / (e - e2) - 1 : 0;
    if (q2 + e2 + long_thres * e2 > q + e + long_thres * e) ++long_thres;
    long_diff = long_thres * (e - e2) - (q2 - q) - e2;

    n_diag = (size_t)qlen + tlen - 1;
    row = (size_t)n_col_ * B;
    if (with_cigar) {
        p = (uint8_t *)calloc(n_diag * row + B, 1);
        if (singletrack) p2 = (uint8_t *)calloc(n_diag * row + B, 1);
        off = (int *)malloc(n_diag * sizeof(int) * 2);
        off_end = off + n_diag;
    }
    /* Same byte layout as the reference's single calloc: u v x y x2 y2 s sf qr,
     * each of tlen_*B bytes except qr; the score fill reads past sf into qr and
     * past qr into zeros, so the layout is part of the semantics. */
    T = (size_t)tlen_ * B;
    mem = (int8_t *)calloc((size_t)tlen_ * 8 * B + (size_t)qlen_ * B + 64 * B + 256, 1);
    u = mem, v = u + T, x = v + T, y = x + T, x2 = y + T, y2 = x2 + T, s = y2 + T;
    sf = (uint8_t *)(s + T), qr = sf + T;
    memset(u, w8(-q - e), T); memset(v, w8(-q - e), T);
    memset(x, w8(-q - e), T); memset(y, w8(-q - e), T);
    memset(x2, w8(-q2 - e2), T); memset(y2, w8(-q2 - e2), T);
    if (!approx_max) {
        H = (int32_t *)malloc(T * 4);
        for (t = 0; t < (int)T; ++t) H[t] = OR_NEG_INF;
    }
    for (t = 0; t < qlen; ++t) qr[t] = query[qlen - 1 - t];
    memcpy(sf, target, (size_t)tlen);

    int8_t *nu = (int8_t *)malloc((size_t)B * 6 + (size_t)B * 2);

    for (r = 0, last_st = last_en = -1; r < qlen + tlen - 1; ++r) {
        if (stop_at >= 0 && stop_interval > 0 && r % stop_interval == 0 && r >= stop_at) {
            ez->stopped = 1;
            break;
        }
        int st = 0, en = tlen - 1, st0, en0, st16, en16, stB, enB, bfirst, blast, b;
        int8_t x1, x21, v1;
        const uint8_t *qrr = qr + (qlen - 1 - r);
        if (st < r - qlen + 1) st = r - qlen + 1;
        if (en > r) en = r;
        if (st < (r - wr + 1) >> 1) st = (r - wr + 1) >> 1;
        if (en > (r + wl) >> 1) en = (r + wl) >> 1;
        if (st > en) { ez->zdropped = 1; break; }
        st0 = st, en0 = en;
        st16 = st0 / 16 * 16, en16 = (en0 + 16) / 16 * 16 - 1;
        stB = st0 / B * B, enB = (en0 + B) / B * B - 1;
        /* boundary cell (r-1, st16-1), ksw2_extd2_avx.c:273-287 */
        if (st16 > 0) {
            if (st16 - 1 >= last_st && st16 - 1 <= last_en)
                x1 = x[st16 - 1], x21 = x2[st16 - 1], v1 = v[st16 - 1];
            else
                x1 = w8(-q - e), x21 = w8(-q2 - e2), v1 = w8(-q - e);
        } else {
            x1 = w8(-q - e), x21 = w8(-q2 - e2);
            v1 = r == 0 ? w8(-q - e) : r < long_thres ? w8(-e) : r == long_thres ? w8(long_diff) : w8(-e2);
        }
        if (en16 >= r) {
            y[r] = w8(-q - e), y2[r] = w8(-q2 - e2);
            u[r] = r == 0 ? w8(-q - e) : r < long_thres ? w8(-e) : r == long_thres ? w8(long_diff) : w8(-e2);
        }
        /* score fill (loop fission); stores whole 16-byte groups past en0 */
        if (!(flag & OR_GENERIC_SC)) {
            for (t = st0; t <= en0; t += B) {
                int lanes = (t + B > en0) ? (en0 - t + 16) / 16 * 16 : B;
                for (int l = 0; l < lanes; ++l) {
                    uint8_t a = sf[t + l], c = qrr[t + l];
                    int8_t sc = a == c ? sc_mch : sc_mis;
                    if (a == (uint8_t)m1 || c == (uint8_t)m1) sc = sc_N;
                    s[t + l] = sc;
                }
            }
        } else {
            for (t = st0; t <= en0; ++t) s[t] = mat[sf[t] * m + qrr[t]];
        }
        if (with_cigar) off[r] = stB, off_end[r] = en16;
        bfirst = stB / B, blast = enB / B;
        int8_t c_x1 = x1, c_x21 = x21, c_v1 = v1;
        for (b = bfirst; b <= blast; ++b) {
            const int base = b * B;
            /* lane that receives the carried (r-1, base+lane-1) value */
            const int blane = (b == bfirst) ? (st16 - base) : 0;
            int8_t *ou = nu, *ov = nu + B, *ox = nu + 2 * B, *oy = nu + 3 * B, *ox2 = nu + 4 * B,
                   *oy2 = nu + 5 * B, *od = nu + 6 * B, *od2 = nu + 7 * B;
            const int8_t nx1 = x[base + B - 1], nx21 = x2[base + B - 1], nv1 = v[base + B - 1];
            const int nstore = (b == blast) ? (en0 - base + 16) / 16 * 16 : B;
            for (int l = 0; l < B; ++l) {
                const int pos = base + l;
                int8_t xs, vs, x2s;
                if (l == blane) xs = c_x1, vs = c_v1, x2s = c_x21;
                else if (l == 0) xs = x[base + 15], vs = v[base + 15], x2s = x2[base + 15]; /* in-block shuffle wrap */
                else xs = x[pos - 1], vs = v[pos - 1], x2s = x2[pos - 1];
                int8_t z = s[pos], ut = u[pos];
                int8_t a = w8(xs + vs), bb = w8(y[pos] + ut), a2 = w8(x2s + vs), b2 = w8(y2[pos] + ut);
                int8_t d = 0;
                if (!with_cigar) {
                    z = max8(z, a); z = max8(z, bb); z = max8(z, a2); z = max8(z, b2);
                    z = min8(z, sc_mch);
                } else if (!(flag & OR_RIGHT)) {
                    d = a > z ? 1 : 0; z = max8(z, a);
                    d = bb > z ? 2 : d; z = max8(z, bb);
                    d = a2 > z ? 3 : d; z = max8(z, a2);
                    d = b2 > z ? 4 : d; z = max8(z, b2);
                    z = min8(z, sc_mch);
                } else {
                    d = z > a ? 0 : 1; z = max8(z, a);
                    d = z > bb ? d : 2; z = max8(z, bb);
                    d = z > a2 ? d : 3; z = max8(z, a2);
                    d = z > b2 ? d : 4; z = max8(z, b2);
                    z = min8(z, sc_mch);
                }
                ou[l] = w8(z - vs);
                ov[l] = w8(z - ut);
                int8_t tq = w8(z - q), tq2 = w8(z - q2);
                a = w8(a - tq), bb = w8(bb - tq), a2 = w8(a2 - tq2), b2 = w8(b2 - tq2);
                ox[l] = w8(max8(a, 0) - (q + e));
                oy[l] = w8(max8(bb, 0) - (q + e));
                ox2[l] = w8(max8(a2, 0) - (q2 + e2));
                oy2[l] = w8(max8(b2, 0) - (q2 + e2));
                if (with_cigar) {
                    if (!(flag & OR_RIGHT)) {
                        d |= a > 0 ? 0x08 : 0; d |= bb > 0 ? 0x10 : 0;
                        d |= a2 > 0 ? 0x20 : 0; d |= b2 > 0 ? 0x40 : 0;
                    } else {
                        d |= a >= 0 ? 0x08 : 0; d |= bb >= 0 ? 0x10 : 0;
                        d |= a2 >= 0 ? 0x20 : 0; d |= b2 >= 0 ? 0x40 : 0;
                    }
                    od[l] = d;
                    od2[l] = ou[l];
                }
            }
            c_x1 = nx1, c_x21 = nx21, c_v1 = nv1;
            for (int l = 0; l < nstore; ++l) {
                const int pos = base + l;
                u[pos] = ou[l], v[pos] = ov[l], x[pos] = ox[l], y[pos] = oy[l];
                x2[pos] = ox2[l], y2[pos] = oy2[l];
                if (with_cigar) {
                    size_t idx = (size_t)r * row + (size_t)(pos - stB);
                    if (singletrack) p[idx] = (uint8_t)ov[l], p2[idx] = (uint8_t)od2[l];
                    else p[idx] = (uint8_t)od[l];
                }
            }
        }
        if (!approx_max) {
            int32_t max_H, max_t;
            if (r > 0) {
                int32_t HH[4], tt[4];
                int en1 = st0 + (en0 - st0) / 4 * 4, i;
                max_H = H[en0] = en0 > 0 ? H[en0 - 1] + u[en0] : H[en0] + v[en0];
                max_t = en0;
                for (i = 0; i < 4; ++i) HH[i] = max_H, tt[i] = max_t - i;
                for (t = st0; t < en1; ++t) {
                    int c = (t - st0) & 3;
                    H[t] += v[t];
                    if (H[t] > HH[c]) HH[c] = H[t], tt[c] = t - c;
                }
                for (i = 0; i < 4; ++i)
                    if (max_H < HH[i]) max_H = HH[i], max_t = tt[i] + i;
                for (; t < en0; ++t) {
                    H[t] += v[t];
                    if (H[t] > max_H) max_H = H[t], max_t = t;
                }
            } else
                H[0] = v[0] - qe, max_H = H[0], max_t = 0;
            if (sse_st) {
                if (en0 == tlen - 1 && H[en0] > ez->mte) ez->mte = H[en0], ez->mte_q = r - ((en0 + 16) / 16 * 16 - 1);
                if (r - st0 == qlen - 1 && H[st0] > ez->mqe) ez->mqe = H[st0], ez->mqe_t = st0;
            } else {
                if (en0 == tlen - 1 && H[en0] >= ez->mte) ez->mte = H[en0], ez->mte_q = r - en0;
                if (r - st0 == qlen - 1 && H[st0] >= ez->mqe) ez->mqe = H[st0], ez->mqe_t = st0;
            }
            if (or_zdrop(ez, max_H, r, max_t, zdrop, e2)) break;
            if (r == qlen + tlen - 2 && en0 == tlen - 1) ez->score = H[tlen - 1];
        } else {
            if (r > 0) {
                if (last_H0_t >= st0 && last_H0_t <= en0 && last_H0_t + 1 >= st0 && last_H0_t + 1 <= en0) {
                    int32_t d0 = v[last_H0_t], d1 = u[last_H0_t + 1];
                    if (d0 > d1) H0 += d0;
                    else H0 += d1, ++last_H0_t;
                } else if (last_H0_t >= st0 && last_H0_t <= en0) {
                    H0 += v[last_H0_t];
                } else {
                    ++last_H0_t, H0 += u[last_H0_t];
                }
            } else
                H0 = v[0] - qe, last_H0_t = 0;
            if ((flag & OR_APPROX_DROP) && or_zdrop(ez, H0, r, last_H0_t, zdrop, e2)) break;
            if (r == qlen + tlen - 2 && en0 == tlen - 1) ez->score = H0;
        }
        last_st = st16, last_en = en16;
    }
    free(nu);
    free(mem);
    free(H);
    if (with_cigar && singletrack) {
        if (!ez->stopped && !ez->zdropped && (sse_st || !(flag & (OR_EXTZ_ONLY | OR_SEMIGLOBAL_END)))) {
            or_singletrack_bt(qlen, query, tlen, target, m, mat, q, e, q2, e2, row, off, off_end,
                              (const int8_t *)p, (const int8_t *)p2, ez);
            if (ez->n_cigar == 0) ez->zdropped = 1;
        } else if (!ez->stopped && !ez->zdropped) {
            ez->zdropped = 1;
        }
    } else if (with_cigar) {
        int rev = !!(flag & OR_REV_CIGAR);
        if (!ez->stopped && !ez->zdropped && (flag & OR_SEMIGLOBAL_END)) {
            if (ez->mqe > ez->mte) {
                ez->score = ez->mqe;
                or_backtrack(rev, p, off, off_end, row, ez->mqe_t, qlen - 1, &ez->m_cigar, &ez->n_cigar, &ez->cigar);
            } else {
                ez->score = ez->mte;
                or_backtrack(rev, p, off, off_end, row, tlen - 1, ez->mte_q, &ez->m_cigar, &ez->n_cigar, &ez->cigar);
            }
        } else if (!ez->stopped && !ez->zdropped && !(flag & OR_EXTZ_ONLY)) {
            or_backtrack(rev, p, off, off_end, row, tlen - 1, qlen - 1, &ez->m_cigar, &ez->n_cigar, &ez->cigar);
        } else if (!ez->zdropped && (flag & OR_EXTZ_ONLY) && ez->mqe + end_bonus > (int)ez->max) {
            ez->reach_end = 1;
            or_backtrack(rev, p, off, off_end, row, ez->mqe_t, qlen - 1, &ez->m_cigar, &ez->n_cigar, &ez->cigar);
        } else if (ez->max_t >= 0 && ez->max_q >= 0) {
            or_backtrack(rev, p, off, off_end, row, ez->max_t, ez->max_q, &ez->m_cigar, &ez->n_cigar, &ez->cigar);
        }
    }
    free(p);
    free(p2);
    free(off);
}

void oracle_free(void *p) { free(p); }
int oracle_sizeof_extz(void) { return (int)sizeof(or_extz_t); }
