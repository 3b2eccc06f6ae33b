// KSW2 extd2, exact anti-diagonal form, on sm_100a: every flag, banded
// (w >= 0), z-drop, approximate max and the Singletrack traceback.
//
// One CTA per pair sweeps the anti-diagonals r = 0 .. qlen+tlen-2 in the
// reference's own array form: int8 cells u, v, x, y, x2, y2 and the score row s
// indexed by target position, recomputed each anti-diagonal over whole SIMD
// blocks [st rounded down to the block, en rounded up to 16] exactly as
// minimap2/ksw2_extd2_avx.c:255-701 (block 64 / 32) and ksw2_extd2_sse.c:136-331
// (block 16) do.  In banded mode the in-band cells read the out-of-band
// padding cells of the previous anti-diagonal, and the traceback may walk into
// them, so the padding lanes are computed here with the same inputs:
//   * stale score-row entries and the score fill's overrun past en0
//     (ksw2_extd2_avx.c:289-311; the fill reads past the target into the
//     reversed query because of the reference's single-allocation layout);
//   * lane 0 of the first block takes its left neighbour from lane 15 of the
//     same block (the in-lane byte shuffle of ksw2_extd2_avx.c:72-84);
//   * int8 wrap-around arithmetic everywhere.
// The exact H row, the 4-class arg-max with its tie-breaks (ksw2_extd2_sse.c:332-367),
// mqe/mte with ">=" (:369-372), z-drop (ksw2.h:201-217), ksw_backtrack with
// off/off_end forcing (ksw2.h:160-192) and the Singletrack reconstruction
// (ksw2_singletrack.cpp:63-176) follow on the device.
#include "ksw2_exact.h"
#include <algorithm>
#include <climits>
#include <mutex>

namespace aw {

namespace {

constexpr int NT = 512;  // threads per CTA (multiple of 64)

struct ExactPair {
    int32_t idx, w;
    int64_t ws_off, TB, row, n_diag;
    int32_t n_col, pad;
};

struct ExactArgs {
    const uint8_t *qcodes, *tcodes;
    const KswPair *pairs;
    const ExactPair *ep;
    uint8_t *ws;
    KswOut *out;
    uint32_t *cig;
    KswScore S;
    int8_t mat[64];
    int m, zdrop, end_bonus, flag, B;
    int stop_interval, stop_at;
    const unsigned long long *deadline;  // the calling thread's deadline word, or null
};

__device__ __forceinline__ int8_t w8(int v) { return (int8_t)(uint8_t)(v & 0xff); }
__device__ __forceinline__ int8_t mx8(int8_t a, int8_t b) { return a > b ? a : b; }
__device__ __forceinline__ int8_t mn8(int8_t a, int8_t b) { return a < b ? a : b; }

struct Ws {
    int8_t *u, *v, *x, *y, *x2, *y2, *s;
    int32_t *H;
    int32_t *off, *off_end;
    uint8_t *p, *p2;
};

__device__ __forceinline__ int64_t al256(int64_t v) { return (v + 255) & ~(int64_t)255; }

__device__ Ws carve(uint8_t *base, const ExactPair &E, bool cigar, bool st) {
    Ws w;
    int64_t o = 0;
    w.u = (int8_t *)base + o; o += E.TB;
    w.v = (int8_t *)base + o; o += E.TB;
    w.x = (int8_t *)base + o; o += E.TB;
    w.y = (int8_t *)base + o; o += E.TB;
    w.x2 = (int8_t *)base + o; o += E.TB;
    w.y2 = (int8_t *)base + o; o += E.TB;
    w.s = (int8_t *)base + o; o += E.TB;
    o = al256(o);
    w.H = (int32_t *)(base + o); o += 4 * E.TB;
    o = al256(o);
    w.off = w.off_end = nullptr;
    w.p = w.p2 = nullptr;
    if (cigar) {
        w.off = (int32_t *)(base + o); o += 4 * E.n_diag;
        w.off_end = (int32_t *)(base + o); o += 4 * E.n_diag;
        o = al256(o);
        w.p = base + o; o += al256(E.n_diag * E.row + 64);
        if (st) w.p2 = base + o;
    }
    return w;
}

// Byte i of the reference's "sf" region and beyond (target codes, zero padding to
// TB, then the reversed query, then zeros): the memory the score fill reads.
__device__ __forceinline__ uint8_t sf_ext(int64_t i, const uint8_t *t, int tlen, const uint8_t *q, int qlen,
                                          int64_t TB) {
    if (i < tlen) return t[i];
    if (i < TB) return 0;
    const int64_t k = i - TB;
    return k < qlen ? q[qlen - 1 - k] : 0;
}
__device__ __forceinline__ uint8_t qr_ext(int64_t k, const uint8_t *q, int qlen) {
    return (k >= 0 && k < qlen) ? q[qlen - 1 - k] : 0;
}

__device__ __forceinline__ int edge8(int r, const KswScore &S) {
    return r == 0 ? -S.qe : r < S.long_thres ? -S.e : r == S.long_thres ? S.long_diff : -S.e2;
}

// (value desc, position asc) arg-max used by the per-class H scan.
__device__ __forceinline__ void amax_first(int &v, int &p, int ov, int op) {
    if (ov > v || (ov == v && op < p)) v = ov, p = op;
}

struct Ez {
    int max, max_q, max_t, mqe, mqe_t, mte, mte_q, score, zdropped, reach_end, stopped;
};

// mte / mqe of a finished anti-diagonal r: with ">=" and mte_q = r - en0 as AnchorWave's
// ksw_extd2 (ksw2_extd2_sse.c:369-372); ksw_extd2_singletrack_sse keeps minimap2's
// strict ">" and mte_q = r - en with en rounded up to its 16-byte block
// (minimap2/ksw2_singletrack.cpp:583-586).
__device__ __forceinline__ void end_rules(Ez &z, const int32_t *H, int r, int st0, int en0, int qlen, int tlen,
                                          bool sse_st) {
    if (sse_st) {
        if (en0 == tlen - 1 && H[en0] > z.mte) z.mte = H[en0], z.mte_q = r - ((en0 + 16) / 16 * 16 - 1);
        if (r - st0 == qlen - 1 && H[st0] > z.mqe) z.mqe = H[st0], z.mqe_t = st0;
    } else {
        if (en0 == tlen - 1 && H[en0] >= z.mte) z.mte = H[en0], z.mte_q = r - en0;
        if (r - st0 == qlen - 1 && H[st0] >= z.mqe) z.mqe = H[st0], z.mqe_t = st0;
    }
}

__device__ bool apply_zdrop(Ez &ez, int H, int r, int t, int zdrop, int e) {
    if (H > ez.max) {
        ez.max = H, ez.max_t = t, ez.max_q = r - t;
    } else if (t >= ez.max_t && r - t >= ez.max_q) {
        const int tl = t - ez.max_t, ql = (r - t) - ez.max_q;
        const int l = tl > ql ? tl - ql : ql - tl;
        if (zdrop >= 0 && ez.max - H > zdrop + l * e) {
            ez.zdropped = 1;
            return true;
        }
    }
    return false;
}

struct Cig {
    uint32_t *buf;
    int n;
    __device__ void push(uint32_t op, int len) {
        if (n > 0 && (buf[n - 1] & 0xf) == op) buf[n - 1] += (uint32_t)len << 4;
        else buf[n++] = (uint32_t)len << 4 | op;
    }
    __device__ void reverse() {
        for (int a = 0, b = n - 1; a < b; ++a, --b) {
            uint32_t t = buf[a];
            buf[a] = buf[b], buf[b] = t;
        }
    }
};

// ksw_backtrack (minimap2/ksw2.h:160-192), rotated layout with off/off_end forcing.
__device__ void backtrack(Cig &c, bool rev, const uint8_t *p, const int32_t *off, const int32_t *off_end,
                          int64_t n_col, int i, int j) {
    int state = 0;
    while (i >= 0 && j >= 0) {
        const int r = i + j;
        int force = -1;
        if (i < off[r]) force = 2;
        if (i > off_end[r]) force = 1;
        const uint32_t tmp = force < 0 ? p[(int64_t)r * n_col + i - off[r]] : 0;
        if (state == 0) state = tmp & 7;
        else if (!(tmp >> (state + 2) & 1)) state = 0;
        if (state == 0) state = tmp & 7;
        if (force >= 0) state = force;
        if (state == 0) c.push(0, 1), --i, --j;
        else if (state == 1 || state == 3) c.push(2, 1), --i;
        else c.push(1, 1), --j;
    }
    if (i >= 0) c.push(2, i + 1);
    if (j >= 0) c.push(1, j + 1);
    if (!rev) c.reverse();
}

__device__ __forceinline__ int st_gap(int l, int o1, int e1, int o2, int e2) {
    if (l <= 0) return 0;
    const long long a = (long long)o1 + (long long)l * e1, b = (long long)o2 + (long long)l * e2;
    return (int)(a > b ? a : b);
}
__device__ __forceinline__ int st_diff(const int8_t *mtx, int i, int j, int64_t n_col, const int32_t *off,
                                       const int32_t *off_end, int o1, int e1, int o2, int e2) {
    if (i < 0 || j < 0) {
        const int c = i < 0 ? j : i;
        return st_gap(c + 1, o1, e1, o2, e2) - st_gap(c, o1, e1, o2, e2);
    }
    const int64_t d = (int64_t)i + j;
    if (i < off[d] || i > off_end[d]) return AW_NEG_INF;
    return (int)mtx[d * n_col + i - off[d]];
}
__device__ __forceinline__ bool st_fin(int v) { return v > AW_NEG_INF / 2 && v < -AW_NEG_INF / 2; }

// ksw2_singletrack_backtrace_affine2p (minimap2/ksw2_singletrack.cpp:63-176).
__device__ bool singletrack_bt(Cig &c, int qlen, const uint8_t *query, int tlen, const uint8_t *target, int m,
                               const int8_t *mat, const KswScore &S, int64_t n_col, const int32_t *off,
                               const int32_t *off_end, const int8_t *p, const int8_t *p2) {
    const int o1 = -S.q, g1 = -S.e, o2 = -S.q2, g2 = -S.e2;
    bool in_m = true;
    int i = tlen - 1, j = qlen - 1, l = 0, dd = 0, di = 0;
    while (i >= 0 && j >= 0) {
        const int dg = i + j;
        if (i < off[dg]) { c.push(1, 1); --j; in_m = true; continue; }
        if (i > off_end[dg]) { c.push(2, 1); --i; in_m = true; continue; }
        if (in_m) {
            const int h = st_diff(p, i, j, n_col, off, off_end, o1, g1, o2, g2);
            const int v = st_diff(p2, i, j - 1, n_col, off, off_end, o1, g1, o2, g2);
            const int cost = mat[target[i] * m + query[j]];
            if (st_fin(h) && st_fin(v) && (long long)h + v == cost) {
                c.push(0, 1);
                --i, --j;
            } else {
                in_m = false, l = 0;
                di = st_diff(p, i, j, n_col, off, off_end, o1, g1, o2, g2);
                dd = st_diff(p2, i, j, n_col, off, off_end, o1, g1, o2, g2);
            }
        } else {
            ++l;
            if (l > i + 1 && l > j + 1) return false;
            const int a1 = o1 + l * g1, a2 = o2 + l * g2, jn = j - l, id = i - l;
            if (id >= -1 && (dd == a1 || dd == a2)) {
                c.push(2, l);
                i = id, in_m = true;
            } else if (jn >= -1 && (di == a1 || di == a2)) {
                c.push(1, l);
                j = jn, in_m = true;
            } else {
                if (jn >= 0) {
                    const int Hh = st_diff(p, i, jn, n_col, off, off_end, o1, g1, o2, g2);
                    di = (st_fin(di) && st_fin(Hh)) ? di + Hh : AW_NEG_INF;
                }
                if (id >= 0) {
                    const int V = st_diff(p2, id, j, n_col, off, off_end, o1, g1, o2, g2);
                    dd = (st_fin(dd) && st_fin(V)) ? dd + V : AW_NEG_INF;
                }
            }
        }
    }
    if (i >= 0) c.push(2, i + 1);
    if (j >= 0) c.push(1, j + 1);
    c.reverse();
    return true;
}

__global__ void __launch_bounds__(NT) ksw_exact_kernel(ExactArgs A) {
    const ExactPair E = A.ep[blockIdx.x];
    const KswPair P = A.pairs[E.idx];
    const KswScore &S = A.S;
    const int tid = threadIdx.x;
    const int qlen = P.qlen, tlen = P.tlen, B = A.B, flag = A.flag;
    const bool with_cigar = !(flag & AW_EZ_SCORE_ONLY);
    const bool approx_max = !!(flag & AW_EZ_APPROX_MAX);
    const bool sse_st = !!(flag & AW_EZ_SSE_SINGLETRACK) && !!(flag & AW_EZ_SINGLETRACK);
    const bool singletrack = (B > 16 || sse_st) && !!(flag & AW_EZ_SINGLETRACK);
    const bool right = !!(flag & AW_EZ_RIGHT);
    const bool generic = !!(flag & AW_EZ_GENERIC_SC);
    const uint8_t *qs = A.qcodes + P.qoff, *ts = A.tcodes + P.toff;
    Ws W = carve(A.ws + E.ws_off, E, with_cigar, singletrack);
    const int8_t sc_mch = A.mat[0], sc_mis = A.mat[1];
    const int m = A.m;
    const int8_t sc_N = A.mat[m * m - 1] == 0 ? w8(-S.e2) : A.mat[m * m - 1];
    const int8_t m1 = (int8_t)(m - 1);
    const int q = S.q, q2 = S.q2, e2 = S.e2, qe = S.qe, qe2 = S.qe2;
    int w = E.w;
    if (w < 0) w = tlen > qlen ? tlen : qlen;
    const int wl = w, wr = w;

    __shared__ int8_t s_carry[2][3];
    __shared__ int s_red_v[NT / 32][4], s_red_p[NT / 32][4];
    __shared__ int s_brk, s_stop;
    __shared__ Ez s_ez;
    __shared__ int s_H0, s_H0t;

    for (int64_t i = tid; i < E.TB; i += NT) {
        W.u[i] = w8(-qe), W.v[i] = w8(-qe), W.x[i] = w8(-qe), W.y[i] = w8(-qe);
        W.x2[i] = w8(-qe2), W.y2[i] = w8(-qe2), W.s[i] = 0;
        W.H[i] = AW_NEG_INF;
    }
    if (tid == 0) {
        s_ez.max = 0, s_ez.max_q = s_ez.max_t = s_ez.mqe_t = s_ez.mte_q = -1;
        s_ez.score = s_ez.mqe = s_ez.mte = AW_NEG_INF;
        s_ez.zdropped = s_ez.reach_end = s_ez.stopped = 0;
        s_brk = 0;
        s_H0 = 0, s_H0t = 0;
    }
    __syncthreads();

    int last_st = -1, last_en = -1;
    const int nd = qlen + tlen - 1;
    const bool polled = A.stop_at >= 0 || A.deadline;
    const int interval = A.stop_interval > 0 ? A.stop_interval : 256;
    for (int r = 0; r < nd; ++r) {
        // ksw_progress_continue (minimap2/ksw2_progress.c:30-38) before anti-diagonal r:
        // a scheduled stop, or the calling thread's deadline, sets ez->stopped
        if (polled && r % interval == 0) {
            if (tid == 0)
                s_stop = (A.stop_at >= 0 && r >= A.stop_at) || aw_deadline_passed(A.deadline);
            __syncthreads();
            if (s_stop) {
                if (tid == 0) s_ez.stopped = 1;
                break;
            }
        }
        int st = 0, en = tlen - 1;
        if (st < r - qlen + 1) st = r - qlen + 1;
        if (en > r) en = r;
        if (st < (r - wr + 1) >> 1) st = (r - wr + 1) >> 1;
        if (en > (r + wl) >> 1) en = (r + wl) >> 1;
        if (st > en) {
            if (tid == 0) s_ez.zdropped = 1;
            break;
        }
        const int st0 = st, en0 = en;
        const int st16 = st0 / 16 * 16, en16 = (en0 + 16) / 16 * 16 - 1;
        const int stB = st0 / B * B;
        // boundary cell (r-1, st16-1); read before this anti-diagonal writes anything
        int8_t x1, x21, v1;
        if (st16 > 0) {
            if (st16 - 1 >= last_st && st16 - 1 <= last_en) x1 = W.x[st16 - 1], x21 = W.x2[st16 - 1], v1 = W.v[st16 - 1];
            else x1 = w8(-qe), x21 = w8(-qe2), v1 = w8(-qe);
        } else {
            x1 = w8(-qe), x21 = w8(-qe2), v1 = w8(edge8(r, S));
        }
        const bool topb = en16 >= r;
        const int64_t qrr0 = (int64_t)qlen - 1 - r;
        // score fill
        if (!generic) {
            const int ngroups = (en0 - st0) / B + 1;
            const int64_t span = (int64_t)ngroups * B;
            for (int64_t o = tid; o < span; o += NT) {
                const int k = (int)(o / B), l = (int)(o % B);
                const int t0 = st0 + k * B;
                const int lanes = (t0 + B > en0) ? (en0 - t0 + 16) / 16 * 16 : B;
                if (l < lanes) {
                    const int64_t pos = t0 + l;
                    const uint8_t a = sf_ext(pos, ts, tlen, qs, qlen, E.TB);
                    const uint8_t c = qr_ext(qrr0 + pos, qs, qlen);
                    int8_t sc = a == c ? sc_mch : sc_mis;
                    if (a == (uint8_t)m1 || c == (uint8_t)m1) sc = sc_N;
                    // past TB the reference's fill lands in its target copy, only at
                    // indices below the current st0, which are never read again
                    if (pos < E.TB) W.s[pos] = sc;
                }
            }
        } else {
            // query base r - pos, through the reversed-query index of the reference's qrr
            for (int pos = st0 + tid; pos <= en0; pos += NT) W.s[pos] = A.mat[ts[pos] * m + qr_ext(qrr0 + pos, qs, qlen)];
        }
        __syncthreads();
        // cells, in NT-wide chunks starting at the block-aligned stB
        int chunk = 0;
        for (int base = stB; base <= en16; base += NT, ++chunk) {
            const int pos = base + tid;
            int8_t nu = 0, nv = 0, nx = 0, ny = 0, nx2 = 0, ny2 = 0, d = 0, pz = 0;
            const bool act = pos <= en16;
            if (act) {
                const int blk = pos / B, l = pos % B, bfirst = stB / B;
                // only the first block takes the band-edge value, at lane st16-stB;
                // lane 0 of every later block takes the previous block's last lane
                int8_t xs, vs, x2s;
                if (blk == bfirst && l == st16 - stB) xs = x1, vs = v1, x2s = x21;
                else if (l == 0 && blk == bfirst) {
                    const int src = blk * B + 15;
                    xs = W.x[src], vs = W.v[src], x2s = W.x2[src];
                } else if (tid == 0) {
                    xs = s_carry[(chunk + 1) & 1][0], vs = s_carry[(chunk + 1) & 1][1], x2s = s_carry[(chunk + 1) & 1][2];
                } else {
                    xs = W.x[pos - 1], vs = W.v[pos - 1], x2s = W.x2[pos - 1];
                }
                int8_t z = W.s[pos];
                int8_t ut, yt, y2t;
                if (topb && pos == r) ut = w8(edge8(r, S)), yt = w8(-qe), y2t = w8(-qe2);
                else ut = W.u[pos], yt = W.y[pos], y2t = W.y2[pos];
                int8_t a = w8(xs + vs), b = w8(yt + ut), a2 = w8(x2s + vs), b2 = w8(y2t + ut);
                if (!with_cigar) {
                    z = mx8(z, a); z = mx8(z, b); z = mx8(z, a2); z = mx8(z, b2);
                } else if (!right) {
                    d = a > z ? 1 : 0; z = mx8(z, a);
                    d = b > z ? 2 : d; z = mx8(z, b);
                    d = a2 > z ? 3 : d; z = mx8(z, a2);
                    d = b2 > z ? 4 : d; z = mx8(z, b2);
                } else {
                    d = z > a ? 0 : 1; z = mx8(z, a);
                    d = z > b ? d : 2; z = mx8(z, b);
                    d = z > a2 ? d : 3; z = mx8(z, a2);
                    d = z > b2 ? d : 4; z = mx8(z, b2);
                }
                z = mn8(z, sc_mch);
                nu = w8(z - vs);
                nv = w8(z - ut);
                pz = nu;
                const int8_t tq = w8(z - q), tq2 = w8(z - q2);
                a = w8(a - tq), b = w8(b - tq), a2 = w8(a2 - tq2), b2 = w8(b2 - tq2);
                nx = w8(mx8(a, 0) - qe);
                ny = w8(mx8(b, 0) - qe);
                nx2 = w8(mx8(a2, 0) - qe2);
                ny2 = w8(mx8(b2, 0) - qe2);
                if (with_cigar) {
                    if (!right) d |= (a > 0 ? 0x08 : 0) | (b > 0 ? 0x10 : 0) | (a2 > 0 ? 0x20 : 0) | (b2 > 0 ? 0x40 : 0);
                    else d |= (a >= 0 ? 0x08 : 0) | (b >= 0 ? 0x10 : 0) | (a2 >= 0 ? 0x20 : 0) | (b2 >= 0 ? 0x40 : 0);
                }
                if (tid == NT - 1) {
                    s_carry[chunk & 1][0] = W.x[pos], s_carry[chunk & 1][1] = W.v[pos], s_carry[chunk & 1][2] = W.x2[pos];
                }
            }
            __syncthreads();
            if (act) {
                W.u[pos] = nu, W.v[pos] = nv, W.x[pos] = nx, W.y[pos] = ny, W.x2[pos] = nx2, W.y2[pos] = ny2;
                if (with_cigar) {
                    const int64_t idx = (int64_t)r * E.row + (pos - stB);
                    if (singletrack) W.p[idx] = (uint8_t)nv, W.p2[idx] = (uint8_t)pz;
                    else W.p[idx] = (uint8_t)d;
                }
            }
        }
        if (with_cigar && tid == 0) W.off[r] = stB, W.off_end[r] = en16;
        __syncthreads();
        if (!approx_max) {
            if (r > 0) {
                if (tid == 0) W.H[en0] = en0 > 0 ? W.H[en0 - 1] + W.u[en0] : W.H[en0] + W.v[en0];
                __syncthreads();
                const int en1 = st0 + (en0 - st0) / 4 * 4;
                int cv[4], cp[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) cv[c] = INT_MIN, cp[c] = INT_MAX;
                for (int t = st0 + tid; t < en0; t += NT) {
                    const int h = W.H[t] + W.v[t];
                    W.H[t] = h;
                    if (t < en1) {
                        const int c = (t - st0) & 3;
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc)
                            if (cc == c) amax_first(cv[cc], cp[cc], h, t);
                    }
                }
#pragma unroll
                for (int c = 0; c < 4; ++c) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const int ov = __shfl_xor_sync(0xffffffffu, cv[c], o), op = __shfl_xor_sync(0xffffffffu, cp[c], o);
                        amax_first(cv[c], cp[c], ov, op);
                    }
                }
                if ((tid & 31) == 0)
                    for (int c = 0; c < 4; ++c) s_red_v[tid >> 5][c] = cv[c], s_red_p[tid >> 5][c] = cp[c];
                __syncthreads();
                if (tid == 0) {
                    for (int wi = 1; wi < NT / 32; ++wi)
                        for (int c = 0; c < 4; ++c) amax_first(cv[c], cp[c], s_red_v[wi][c], s_red_p[wi][c]);
                    int max_H = W.H[en0], max_t = en0;
                    for (int c = 0; c < 4; ++c)
                        if (cp[c] != INT_MAX && max_H < cv[c]) max_H = cv[c], max_t = cp[c];
                    for (int t = en1; t < en0; ++t)
                        if (W.H[t] > max_H) max_H = W.H[t], max_t = t;
                    Ez &z = s_ez;
                    end_rules(z, W.H, r, st0, en0, qlen, tlen, sse_st);
                    if (apply_zdrop(z, max_H, r, max_t, A.zdrop, e2)) s_brk = 1;
                    else if (r == qlen + tlen - 2 && en0 == tlen - 1) z.score = W.H[tlen - 1];
                }
            } else if (tid == 0) {
                W.H[0] = W.v[0] - S.qe_pre;
                Ez &z = s_ez;
                const int max_H = W.H[0], max_t = 0;
                end_rules(z, W.H, r, st0, en0, qlen, tlen, sse_st);
                if (apply_zdrop(z, max_H, r, max_t, A.zdrop, e2)) s_brk = 1;
                else if (r == qlen + tlen - 2 && en0 == tlen - 1) z.score = W.H[tlen - 1];
            }
        } else if (tid == 0) {
            int H0 = s_H0, lt = s_H0t;
            if (r > 0) {
                if (lt >= st0 && lt <= en0 && lt + 1 >= st0 && lt + 1 <= en0) {
                    const int d0 = W.v[lt], d1 = W.u[lt + 1];
                    if (d0 > d1) H0 += d0;
                    else H0 += d1, ++lt;
                } else if (lt >= st0 && lt <= en0) {
                    H0 += W.v[lt];
                } else {
                    ++lt, H0 += W.u[lt];
                }
            } else
                H0 = W.v[0] - S.qe_pre, lt = 0;
            s_H0 = H0, s_H0t = lt;
            if ((flag & AW_EZ_APPROX_DROP) && apply_zdrop(s_ez, H0, r, lt, A.zdrop, e2)) s_brk = 1;
            else if (r == qlen + tlen - 2 && en0 == tlen - 1) s_ez.score = H0;
        }
        __syncthreads();
        if (s_brk) break;
        last_st = st16, last_en = en16;
    }
    __syncthreads();
    if (tid != 0) return;
    Ez z = s_ez;
    int n_cigar = 0;
    if (with_cigar) {
        Cig c{A.cig + P.cig_off, 0};
        const int64_t n_col = E.row;
        if (singletrack) {
            // ksw_extd2_singletrack_sse reconstructs whatever the EXTZ/SEMIGLOBAL flags
            // (minimap2/ksw2_singletrack.cpp:606-615)
            if (!z.stopped && !z.zdropped && (sse_st || !(flag & (AW_EZ_EXTZ_ONLY | AW_EZ_SEMIGLOBAL_END)))) {
                const bool ok = singletrack_bt(c, qlen, qs, tlen, ts, m, A.mat, S, n_col, W.off, W.off_end,
                                               (const int8_t *)W.p, (const int8_t *)W.p2);
                if (!ok) c.n = 0;
                if (c.n == 0) z.zdropped = 1;
            } else if (!z.stopped && !z.zdropped) {
                z.zdropped = 1;
            }
        } else {
            const bool rev = !!(flag & AW_EZ_REV_CIGAR);
            if (!z.stopped && !z.zdropped && (flag & AW_EZ_SEMIGLOBAL_END)) {
                if (z.mqe > z.mte) {
                    z.score = z.mqe;
                    backtrack(c, rev, W.p, W.off, W.off_end, n_col, z.mqe_t, qlen - 1);
                } else {
                    z.score = z.mte;
                    backtrack(c, rev, W.p, W.off, W.off_end, n_col, tlen - 1, z.mte_q);
                }
            } else if (!z.stopped && !z.zdropped && !(flag & AW_EZ_EXTZ_ONLY)) {
                backtrack(c, rev, W.p, W.off, W.off_end, n_col, tlen - 1, qlen - 1);
            } else if (!z.zdropped && (flag & AW_EZ_EXTZ_ONLY) && z.mqe + A.end_bonus > z.max) {
                z.reach_end = 1;
                backtrack(c, rev, W.p, W.off, W.off_end, n_col, z.mqe_t, qlen - 1);
            } else if (z.max_t >= 0 && z.max_q >= 0) {
                backtrack(c, rev, W.p, W.off, W.off_end, n_col, z.max_t, z.max_q);
            }
        }
        n_cigar = c.n;
    }
    KswOut o;
    o.score = z.score, o.max = z.max, o.max_q = z.max_q, o.max_t = z.max_t;
    o.mqe = z.mqe, o.mqe_t = z.mqe_t, o.mte = z.mte, o.mte_q = z.mte_q;
    o.n_cigar = n_cigar, o.zdropped = z.zdropped, o.reach_end = z.reach_end, o.stopped = z.stopped;
    A.out[E.idx] = o;
}

std::mutex g_mu;
int g_block = 64;
// thread-local like the reference's callback state (ksw2_progress.c:11-13)
thread_local int t_stop_interval = 0, t_stop_at = -1;

int64_t host_al256(int64_t v) { return (v + 255) & ~(int64_t)255; }

}  // namespace

int exact_block() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_block;
}
void set_exact_block(int b) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (b == 16 || b == 32 || b == 64) g_block = b;
}
void set_exact_stop(int interval, int stop_at) {
    t_stop_interval = interval > 0 ? interval : 1;
    t_stop_at = stop_at < 0 ? -1 : stop_at;
}
bool exact_stop_enabled() { return t_stop_at >= 0; }

int run_exact_ksw(size_t n_exact, const int32_t *d_ids, const uint8_t *d_q, const uint8_t *d_t,
                  const KswPair *d_pairs, const std::vector<KswPair> &h_pairs, const std::vector<int32_t> &ids,
                  const std::vector<int> &w, int m, const int8_t *mat, const KswScore &S, int zdrop, int end_bonus,
                  int flag, KswOut *d_out, uint32_t *d_cig, DevBuf &ws, cudaStream_t st, int *launches,
                  const unsigned long long *deadline) {
    (void)d_ids;
    if (n_exact == 0) return 0;
    int B;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        B = g_block;
    }
    // ksw_extd2_singletrack_sse works on 16-byte blocks whatever the host's ISA
    const bool sse_st = (flag & AW_EZ_SSE_SINGLETRACK) && (flag & AW_EZ_SINGLETRACK);
    if (sse_st) B = 16;
    const int stop_interval = t_stop_interval, stop_at = t_stop_at;
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY);
    const bool stk = (B > 16 || sse_st) && (flag & AW_EZ_SINGLETRACK);
    // per-pair workspace sizes
    std::vector<ExactPair> eps;
    std::vector<int64_t> sizes;
    for (int32_t i : ids) {
        const KswPair &P = h_pairs[i];
        ExactPair E;
        E.idx = i;
        E.w = w[i];
        int ww = E.w < 0 ? std::max(P.qlen, P.tlen) : E.w;
        const int tlen_ = (P.tlen + B - 1) / B;
        int n_col = std::min(P.qlen, P.tlen);
        n_col = ((n_col < ww + 1 ? n_col : ww + 1) + B - 1) / B + 1;
        E.TB = (int64_t)tlen_ * B;
        E.row = (int64_t)n_col * B;
        E.n_col = n_col;
        E.n_diag = (int64_t)P.qlen + P.tlen - 1;
        E.pad = 0;
        int64_t sz = host_al256(7 * E.TB) + host_al256(4 * E.TB);
        if (cigar) {
            sz += host_al256(8 * E.n_diag);
            sz += host_al256(E.n_diag * E.row + 64) * (stk ? 2 : 1);
        }
        E.ws_off = 0;
        eps.push_back(E);
        sizes.push_back(host_al256(sz));
    }
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = (size_t)8 << 30;
    const int64_t budget = std::max<int64_t>((int64_t)(fr * 0.5) + (int64_t)ws.cap, (int64_t)1 << 28);
    // groups of pairs whose workspaces fit the budget together
    size_t a = 0;
    while (a < eps.size()) {
        int64_t used = host_al256(sizeof(ExactPair) * eps.size());
        size_t b = a;
        while (b < eps.size() && (b == a || used + sizes[b] <= budget) && b - a < 4096) {
            eps[b].ws_off = used;
            used += sizes[b];
            ++b;
        }
        if (used > budget) {
            set_error("exact KSW2 workspace exceeds the device memory budget");
            return AW_E_NOMEM_INTERNAL;
        }
        cudaError_t ce = ws.ensure((size_t)used);
        if (ce != cudaSuccess) {
            set_error("cudaMalloc of the exact KSW2 workspace failed");
            return AW_E_NOMEM_INTERNAL;
        }
        ExactPair *d_ep = (ExactPair *)ws.p;
        if (cudaMemcpyAsync(d_ep, eps.data() + a, sizeof(ExactPair) * (b - a), cudaMemcpyHostToDevice, st) !=
            cudaSuccess) {
            set_error("copy of exact-kernel descriptors failed");
            return AW_E_CUDA_INTERNAL;
        }
        ExactArgs A;
        A.qcodes = d_q, A.tcodes = d_t, A.pairs = d_pairs, A.ep = d_ep, A.ws = (uint8_t *)ws.p;
        A.out = d_out, A.cig = d_cig, A.S = S;
        memset(A.mat, 0, sizeof(A.mat));
        memcpy(A.mat, mat, (size_t)m * m);
        A.m = m, A.zdrop = zdrop, A.end_bonus = end_bonus, A.flag = flag, A.B = B;
        A.stop_interval = stop_interval, A.stop_at = stop_at, A.deadline = deadline;
        ksw_exact_kernel<<<(unsigned)(b - a), NT, 0, st>>>(A);
        if (cudaGetLastError() != cudaSuccess) {
            set_error("exact KSW2 kernel launch failed");
            return AW_E_CUDA_INTERNAL;
        }
        if (launches) ++*launches;
        // the descriptor copy of the next group must not overtake this launch
        if (b < eps.size() && cudaStreamSynchronize(st) != cudaSuccess) {
            set_error("exact KSW2 kernel failed");
            return AW_E_CUDA_INTERNAL;
        }
        a = b;
    }
    return 0;
}

}  // namespace aw
