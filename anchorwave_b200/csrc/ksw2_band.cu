// KSW2 extd2, banded form (w >= 0) and the Singletrack traceback, on sm_100a.
//
// The reference sweeps anti-diagonals r and keeps the int8 difference cells in
// arrays indexed by target position t; on each anti-diagonal it recomputes whole
// SIMD blocks [stB, en16] (st0 rounded down to the block, en0 rounded up to 16),
// so cells just outside the band ("padding") are computed from whatever the arrays
// held, and the in-band cells and the traceback read them
// (minimap2/ksw2_extd2_avx.c:255-701, ksw2_extd2_sse.c:136-331).  This kernel
// computes the same cells in target-column strips swept row by row (the layout of
// the full-matrix kernel) and restates the array semantics cell by cell:
//   * a column's registers hold the last value written at its position, so a
//     column that is not computed on a row keeps its previous values;
//   * left input of cell (t, j): the cell (t-1, j) if it was computed, else the
//     array's initial values; at t == st16 the reference's boundary value
//     (x[st16-1] only on the anti-diagonal where st16 advanced, constants
//     otherwise, the matrix edge when st16 == 0, ksw2_extd2_avx.c:273-287); at
//     t == stB < st16 (lane 0 of the first block) the in-register wrap to lane 15,
//     i.e. cell (stB+15, j-16), kept in a 16-row shared-memory ring;
//   * up input: the column registers, the top-edge values on row 0;
//   * score: the score-fill (ksw2_extd2_avx.c:289-311) refreshes position t on
//     anti-diagonal r when st0 <= t <= st0+16*ceil((en0-st0+1)/16)-1 (en0 for
//     generic scoring); otherwise the stale value of the last fill stays;
//   * H row: H[t] += v[t] inside the band, H[en0] = H[en0-1] + u[en0] on the right
//     edge (ksw2_extd2_sse.c:332-367), mqe/mte with ">=" (:369-372), the score
//     on the last anti-diagonal; the anti-diagonal loop stops at the first empty
//     band (:151-154, zdropped = 1).
// Rows above the matrix (j < 0) only refresh the stale score; rows below it and
// columns right of it never reach a cell of the matrix.  Rows where a lane's 8
// cells all lie strictly inside the band take the full-matrix cell arithmetic
// unchanged (the fast path); the rest go through the per-cell rules above.
//
// Work decomposition: every (pair, strip) is a unit of a device queue, ordered so
// that a strip is always taken after the strip on its left; a warp takes a unit,
// waits (bounded) for the left strip's published rows in global memory and sweeps
// its rows with the one-row lane skew of the full-matrix kernel.  Many warps,
// across CTAs, work on one pair at once, so a single long interval fills the GPU.
#include "ksw2_band.h"
#include "tb_walk.cuh"

#include <algorithm>
#include <climits>
#include <cstring>
#include <cuda/atomic>

namespace aw {

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct Geom {
    int qlen, tlen, w, nd, rb, bmask;  // bmask = ~(block - 1)
    __device__ __forceinline__ int st0(int r) const { return max(max(0, r - qlen + 1), (r - w + 1) >> 1); }
    __device__ __forceinline__ int en0(int r) const { return min(min(tlen - 1, r), (r + w) >> 1); }
};

__device__ __forceinline__ int prmt_sx(uint32_t lo, uint32_t hi, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return (int)r;
}
__device__ __forceinline__ int sx8(uint32_t w) { return (int)(int8_t)(uint8_t)w; }
__device__ __forceinline__ uint32_t pack3(int a, int b, int c, uint32_t top) {
    return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) | (top << 24);
}
__device__ __forceinline__ int edge_diff(int r, const KswScore &S) {
    return r == 0 ? -S.qe : r < S.long_thres ? -S.e : r == S.long_thres ? S.long_diff : -S.e2;
}

// One cell of the reference recurrence in 32-bit registers (the host routes only
// parameter sets whose int8 intermediates cannot wrap).  xs/vs/x2s: left input in,
// this cell's x/v/x2 out; ut/yt/y2t: up input in, this cell's u/y/y2 out.
template <bool ARGMAX, bool RIGHT>
__device__ __forceinline__ void cell(int s, int &xs, int &vs, int &x2s, int &ut, int &yt, int &y2t, int &d,
                                     const KswScore &S) {
    const int a = xs + vs, b = yt + ut, a2 = x2s + vs, b2 = y2t + ut;
    int z = s;
    if (!ARGMAX) {
        z = __vimax3_s32(z, a, b);
        z = __vimax3_s32(z, a2, b2);
    } else {
        // arg-max by priority tags in the low 4 bits of 16 * candidate: the larger tag wins a
        // tie of values, so the max gives z and the state code at once.  Left-aligned: the
        // first candidate wins a tie (ksw2_extd2_sse.c:244-251), tags s=7 > a=6 > ... > b2=3,
        // code = tag ^ 7; right-aligned: the last (:291-298), tags = codes 0..4.
        constexpr int Ts = RIGHT ? 0 : 7, Ta = RIGHT ? 1 : 6, Tb = RIGHT ? 2 : 5, Ta2 = RIGHT ? 3 : 4,
                      Tb2 = RIGHT ? 4 : 3;
        int zt = __vimax3_s32(s * 16 + Ts, b * 16 + Tb, b2 * 16 + Tb2);
        zt = __vimax3_s32(zt, a * 16 + Ta, a2 * 16 + Ta2);
        d = RIGHT ? (zt & 15) : ((zt & 15) ^ 7);
        z = zt >> 4;
    }
    z = min(z, S.mch);
    const int un = z - vs, vn = z - ut;
    if (!(ARGMAX && RIGHT)) {
        const int nez = -S.e - z, nez2 = -S.e2 - z;
        xs = __viaddmax_s32(a, nez, -S.qe);
        yt = __viaddmax_s32(b, nez, -S.qe);
        x2s = __viaddmax_s32(a2, nez2, -S.qe2);
        y2t = __viaddmax_s32(b2, nez2, -S.qe2);
        if (ARGMAX) {
            d += 0x08 * __viaddmin_s32(xs, S.qe, 1);
            d += 0x10 * __viaddmin_s32(yt, S.qe, 1);
            d += 0x20 * __viaddmin_s32(x2s, S.qe2, 1);
            d += 0x40 * __viaddmin_s32(y2t, S.qe2, 1);
        }
    } else {
        const int aa = a - z + S.q, bb = b - z + S.q, aa2 = a2 - z + S.q2, bb2 = b2 - z + S.q2;
        xs = max(aa, 0) - S.qe;
        yt = max(bb, 0) - S.qe;
        x2s = max(aa2, 0) - S.qe2;
        y2t = max(bb2, 0) - S.qe2;
        d |= (aa >= 0 ? 0x08 : 0) | (bb >= 0 ? 0x10 : 0) | (aa2 >= 0 ? 0x20 : 0) | (bb2 >= 0 ? 0x40 : 0);
    }
    ut = un;
    vs = vn;
}

// The Singletrack tracks (v, u) instead of the state bytes: the Singletrack entries of
// the AVX builds (blocks of 32 or 64 bytes), and ksw_extd2_singletrack_sse (16-byte blocks).
bool singletrack_tracks(int flag, int block) {
    return (flag & AW_EZ_SINGLETRACK) && (block > 16 || (flag & AW_EZ_SSE_SINGLETRACK));
}

__device__ __forceinline__ unsigned long long end_key(int v, int pos) {
    return ((unsigned long long)((uint32_t)v ^ 0x80000000u) << 32) | (uint32_t)pos;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct BandArgs {
    const uint8_t *qcodes, *tcodes;
    const BandPairDev *pairs;
    const BandStripDev *strips;
    const int2 *units;
    int32_t n_units;
    int32_t *queue, *progress, *error;
    uint8_t *tb;
    uint2 *bnd;
    BandRes *res;
    KswScore sc;
    int block, generic;
    // ksw_extd2_singletrack_sse's end rules: strict ">" for mqe/mte (the earliest position
    // wins a tie; minimap2/ksw2_singletrack.cpp:583-586)
    int sse_st;
    int store_ckpt;  // 1: store the traceback of recomputed pairs too (their group passes)
    const unsigned long long *deadline;  // null: no deadline
    // recompute rounds: the pairs' walk states; a round's strips stop at the row the walk has
    // reached (it only moves up and left), strips of a finished walk compute nothing
    const BandWalkState *walk;
};

constexpr uint64_t WAIT_NS = 20ull * 1000 * 1000 * 1000;  // bounded wait on the left strip
// rows per publication of a strip's boundary column: the strip on the right starts a row once
// the PUB rows from it are published (lane 31 finishes row j 31 steps after lane 0), so a hop
// between strips costs strip width + 31 + PUB lane-steps
constexpr int PUB = 8;

// NC target columns per lane (strips of 32*NC columns): 8 for throughput, 4 for a shorter
// pipeline lag between strips when few long pairs run.
template <bool CIGAR, bool RIGHT, bool ST, int NC>
__global__ void __launch_bounds__(256, 2) ksw_band_kernel(BandArgs A) {
    constexpr int C = NC;
    // ARGMAX: the state byte is stored (CIGAR without Singletrack)
    constexpr bool ARGMAX = CIGAR && !ST;
    constexpr int CB = ST ? 2 * C : C;  // traceback bytes per lane-step
    // the block wrap reads column stB+15: lane +D of the stB lane, its last column
    constexpr int D = 16 / C - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t ring[8][16][32];
    const KswScore &S = A.sc;
    const int B = A.block;
    const bool src_lane = B > 16 && lane >= D && (((lane - D) * C) & (B - 1)) == 0;

    for (;;) {
        int u = 0;
        if (lane == 0) u = atomicAdd(A.queue, 1);
        u = __shfl_sync(FULL, u, 0);
        if (u >= A.n_units) break;
        const int2 un = A.units[u];
        const BandPairDev P = A.pairs[un.x];
        const int s = un.y;
        const BandStripDev St = A.strips[P.strip0 + s];
        // the last row this pass needs: the strip's last band row, or in a recompute round the
        // walk's row (the same limit for every strip of the pair, producers included)
        int wlim = INT_MAX;
        if (A.walk) {
            const BandWalkState wk = A.walk[un.x];
            wlim = wk.done ? -1 : wk.j;
        }
        const int jstart = St.jstart, jlo = St.jlo, jend = min(St.jend, wlim);
        if (jend < jlo) continue;  // nothing of this strip is computed
        volatile int32_t *stop_word = &A.res[un.x].stopped;
        if (A.deadline && *stop_word) continue;  // the pair stopped at the deadline
        const Geom g{P.qlen, P.tlen, P.w, P.qlen + P.tlen - 1, P.rb, ~(B - 1)};
        const int qlen = P.qlen, tlen = P.tlen, qm1 = qlen - 1, tm1 = tlen - 1;
        const int rlim = min(g.nd, g.rb);
        const uint8_t *qs = A.qcodes + P.qoff, *ts = A.tcodes + P.toff;
        const int col0 = s * 32 * C + lane * C;
        const bool last_strip = s + 1 == P.nstrip;
        // the strip on the left: its published rows and its final H (an empty strip
        // computes nothing, so its column keeps the initial values)
        int prod_lo = 0, prod_hi = -1;
        const uint2 *bnd_prod = nullptr;
        int32_t *prog_prod = nullptr;
        if (s > 0) {
            const BandStripDev Pr = A.strips[P.strip0 + s - 1];
            if (min(Pr.jend, wlim) >= Pr.jlo) {
                prod_lo = Pr.jlo, prod_hi = min(Pr.jend, wlim);
                bnd_prod = A.bnd + Pr.bnd_off;
                prog_prod = A.progress + PROG_STRIDE * (P.strip0 + s - 1);
            }
        }
        uint2 *bnd_me = A.bnd + St.bnd_off;
        int32_t *prog_me = A.progress + PROG_STRIDE * (P.strip0 + s);
        uint8_t *tbp = CIGAR ? A.tb + St.tb_off : nullptr;
        const bool store_tb = CIGAR && (!P.ckpt || A.store_ckpt);  // this strip's traceback is kept
        BandRes *R = A.res + un.x;
        // lane constants of the closed-form bounds: floor16 and the block end of the lane's columns
        const int F16 = col0 & ~15, XB = (col0 & g.bmask) + B - 1;

        int ut[C], yt[C], y2t[C], H[C];
        uint32_t rlo[C], rhi[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const int t = col0 + c;
            const int tc = t < tlen ? (ts[t] & 7) : 0;
            rlo[c] = S.tab_lo[tc];
            rhi[c] = S.tab_hi[tc];
            ut[c] = -S.qe, yt[c] = -S.qe, y2t[c] = -S.qe2;
            H[c] = AW_NEG_INF;
        }
        uint32_t sreg0 = 0, sreg1 = 0;  // stale score bytes of columns 0-3 / 4-7
        int lastfast = INT_MIN;          // row of the latest fast step (all 8 scores fresh there)
        const uint32_t init_pack = pack3(-S.qe, -S.qe, -S.qe2, 0);
        uint32_t carry = 0, qchunk = 0;
        int Hcarry = AW_NEG_INF;
        uint2 bchunk = make_uint2(init_pack, (uint32_t)AW_NEG_INF);
        int seen = INT_MIN;  // lane 0: the left strip's progress count last read
        bool failed = false;
        const int nsteps = jend - jstart + 32;
        for (int k = 0; k < nsteps; ++k) {
            if ((k & 31) == 0 && A.deadline) {
                // cooperative stop, polled every 32 rows (ksw2_progress.c:30-38 polls every
                // 256 anti-diagonals); the pair's other strips see the flag and stop too
                int st = 0;
                if (lane == 0) {
                    st = *stop_word;
                    if (!st && aw_deadline_passed(A.deadline)) st = 1, atomicExch((int32_t *)stop_word, 1);
                }
                if (__shfl_sync(FULL, st, 0)) break;
            }
            if ((k & 31) == 0) {
                const int J = jstart + k, jr = J + lane;
                qchunk = (jr >= 0 && jr < qlen) ? qs[jr] : 0u;
            }
            if (prog_prod && (k & (PUB - 1)) == 0) {
                // rows J..J+PUB-1 of the left strip (published rows, or past its last row its
                // final H with the initial x/v/x2), loaded by the lanes that hold them in the
                // 32-row chunk the step shuffles from (lane L holds row jstart + (k & ~31) + L)
                const int J = jstart + k, jr = jstart + (k & ~31) + lane;
                const int need = J + PUB - 1 > prod_hi ? prod_hi + 2 : J + PUB;
                if (J + PUB - 1 >= prod_lo && lane == 0 && seen < need) {
                    // one poller per warp with back-off; the bound and the error flag
                    // (another warp gave up) are checked every 32 polls
                    cuda::atomic_ref<int32_t, cuda::thread_scope_device> pr(*prog_prod);
                    seen = pr.load(cuda::memory_order_acquire);
                    if (seen < need) {
                        const uint64_t t0 = globaltimer();
                        unsigned ns = 32, polls = 0;
                        while ((seen = pr.load(cuda::memory_order_acquire)) < need) {
                            __nanosleep(ns);
                            ns = ns < 1024 ? ns * 2 : ns;
                            if (A.deadline && *stop_word) break;  // the left strip stopped
                            if ((++polls & 31) == 0 &&
                                (globaltimer() - t0 > WAIT_NS || *(volatile int32_t *)A.error)) {
                                failed = true;
                                break;
                            }
                        }
                    }
                }
                failed = __shfl_sync(FULL, failed, 0);
                if (failed) {
                    if (lane == 0) atomicExch(A.error, 1);
                    break;
                }
                if (A.deadline && __shfl_sync(FULL, lane == 0 ? *stop_word : 0, 0)) break;
                if ((lane & ~(PUB - 1)) == (k & 31)) {
                    if (jr >= prod_lo && jr <= prod_hi) bchunk = __ldcg(bnd_prod + (jr - prod_lo));
                    else if (jr > prod_hi) bchunk = make_uint2(init_pack, __ldcg(bnd_prod + (prod_hi - prod_lo + 1)).y);
                    else bchunk = make_uint2(init_pack, (uint32_t)AW_NEG_INF);
                }
            }
            const uint32_t qv = __shfl_sync(FULL, qchunk, k & 31);
            const uint32_t bx = __shfl_sync(FULL, bchunk.x, k & 31);
            const int bh = (int)__shfl_sync(FULL, bchunk.y, k & 31);
            const uint32_t in = __shfl_up_sync(FULL, carry, 1);
            const int Hin = __shfl_up_sync(FULL, Hcarry, 1);
            const int j = jstart + k - lane;
            int xs, vs, x2s, Hl;
            uint32_t qc;
            if (lane == 0) {
                qc = qv;
                if (s == 0) xs = -S.qe, vs = edge_diff(j, S), x2s = -S.qe2, Hl = AW_NEG_INF;
                else xs = sx8(bx), vs = sx8(bx >> 8), x2s = sx8(bx >> 16), Hl = bh;
            } else {
                qc = in >> 24;
                xs = sx8(in), vs = sx8(in >> 8), x2s = sx8(in >> 16), Hl = Hin;
            }
            const bool active = j >= jstart && j <= jend;
            const int r0 = col0 + j;
            // all 8 cells strictly inside the band, with natural neighbours: the fast path
            const bool fast = active && j > 0 && col0 > g.st0(r0) && col0 + C - 1 < g.en0(r0 + C - 1) &&
                              r0 + C - 1 < rlim;
            // one path for the whole warp, so an edge step costs the edge code once
            const bool warp_fast = __all_sync(FULL, fast || !active);
            uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;  // traceback bytes of this lane-step
            if (active) {
                if (warp_fast && ARGMAX && !store_tb) {
                    // no traceback is kept for this strip (a recomputed pair's first pass, or a
                    // pair whose band empties): the cells without their state bytes
                    const uint32_t sel = qc * 0x1111u + 0x8880u;
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        int d = 0;
                        const int sc = prmt_sx(rlo[c], rhi[c], sel);
                        cell<false, RIGHT>(sc, xs, vs, x2s, ut[c], yt[c], y2t[c], d, S);
                        H[c] += vs;
                    }
                    lastfast = j;
                    carry = pack3(xs, vs, x2s, qc);
                    Hcarry = H[C - 1];
                } else if (warp_fast) {
                    const uint32_t sel = qc * 0x1111u + 0x8880u;
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        int d = 0;
                        const int sc = prmt_sx(rlo[c], rhi[c], sel);
                        cell<ARGMAX, RIGHT>(sc, xs, vs, x2s, ut[c], yt[c], y2t[c], d, S);
                        H[c] += vs;
                        if (ARGMAX) {
                            if (c < 4) w0 |= (uint32_t)d << (8 * c);
                            else w1 |= (uint32_t)d << (8 * (c - 4));
                        } else if (ST) {
                            if (c < 4) w0 |= (uint32_t)(vs & 0xff) << (8 * c), w2 |= (uint32_t)(ut[c] & 0xff) << (8 * c);
                            else w1 |= (uint32_t)(vs & 0xff) << (8 * (c - 4)), w3 |= (uint32_t)(ut[c] & 0xff) << (8 * (c - 4));
                        }
                    }
                    lastfast = j;
                    carry = pack3(xs, vs, x2s, qc);
                    Hcarry = H[C - 1];
                } else {
                    if (lastfast != INT_MIN) {
                        // the fast steps refreshed every score of this lane; rebuild the stale bytes
                        const uint32_t sl = (uint32_t)qs[lastfast] * 0x1111u + 0x8880u;
                        sreg0 = sreg1 = 0;
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const uint32_t b = (uint32_t)prmt_sx(rlo[c], rhi[c], sl) & 0xffu;
                            if (c < 4) sreg0 |= b << (8 * c);
                            else sreg1 |= b << (8 * (c - 4));
                        }
                        lastfast = INT_MIN;
                    }
                    const uint32_t selj = (j < 0 ? 0u : qc) * 0x1111u + 0x8880u;
                    int fx = xs, fv = vs, fx2 = x2s, Hf = Hl;
                    if (j < 0) {
                        // above the matrix: only the score fill of the reference runs here
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const int t = col0 + c, r = r0 + c;
                            if (t <= tm1 && r >= 0 && r < rlim) {
                                const int st0 = g.st0(r), en0 = g.en0(r);
                                const int fe = A.generic ? en0 : st0 + ((en0 - st0 + 16) & ~15) - 1;
                                if (st0 <= t && t <= fe) {
                                    const uint32_t b = (uint32_t)prmt_sx(rlo[c], rhi[c], selj) & 0xffu;
                                    if (c < 4) sreg0 = (sreg0 & ~(0xffu << (8 * c))) | (b << (8 * c));
                                    else sreg1 = (sreg1 & ~(0xffu << (8 * (c - 4)))) | (b << (8 * (c - 4)));
                                }
                            }
                        }
                        fx = -S.qe, fv = -S.qe, fx2 = -S.qe2, Hf = H[C - 1];
                    } else {
                        // Closed forms of the per-cell geometry over this lane-step (cell c: t = col0+c,
                        // r = r0+c): in band  <=> cB <= c <= cE;  computed (stB <= t <= en16) <=>
                        // cRlo <= c <= cRhi;  right band edge (t == en0) <=> in band and
                        // (t == tlen-1 or j == 0 or t >= j+w-1).
                        const int cB = max(0, j - g.w - col0);
                        const int cE = min(min(tm1 - col0, j + g.w - col0), min(rlim - 1 - r0, C - 1));
                        const int cRlo = max(0, 2 * F16 - col0 - j - g.w);
                        const int cRhi = min(min(XB + qm1 - r0, 2 * XB + g.w - r0), min(min(tm1 - col0, rlim - 1 - r0), C - 1));
                        const int redge = j + g.w - 1 - col0;  // c >= redge: t >= j+w-1
                        // the band-edge lane st16 and the block wrap stB can only be column col0 (c = 0)
                        if (r0 < rlim) {
                            const int st0 = g.st0(r0), st16 = st0 & ~15, stB = st0 & g.bmask;
                            if (col0 == st16) {
                                if (st16 == 0) fx = -S.qe, fv = edge_diff(j, S), fx2 = -S.qe2;
                                else if ((g.st0(r0 - 1) & ~15) == st16) fx = -S.qe, fv = -S.qe, fx2 = -S.qe2;
                            } else if (col0 == stB) {
                                const uint32_t wv = ring[warp][(k + D) & 15][lane + D];
                                fx = sx8(wv), fv = sx8(wv >> 8), fx2 = sx8(wv >> 16);
                            }
                        }
                        // score fill right of the band (st0 <= t <= fe, fe <= en0+15 <= (r+w)/2+15,
                        // i.e. t <= j+w+30): per cell, in the lanes that reach it
                        if (cE < C - 1 && col0 + cE + 1 <= j + g.w + 30) {
#pragma unroll
                            for (int c = 0; c < C; ++c) {
                                const int t = col0 + c, r = r0 + c;
                                if (c > cE && t <= tm1 && r < rlim) {
                                    const int st0 = g.st0(r), en0 = g.en0(r);
                                    const int fe = A.generic ? en0 : st0 + ((en0 - st0 + 16) & ~15) - 1;
                                    if (t <= fe) {
                                        const uint32_t b = (uint32_t)prmt_sx(rlo[c], rhi[c], selj) & 0xffu;
                                        if (c < 4) sreg0 = (sreg0 & ~(0xffu << (8 * c))) | (b << (8 * c));
                                        else sreg1 = (sreg1 & ~(0xffu << (8 * (c - 4)))) | (b << (8 * (c - 4)));
                                    }
                                }
                            }
                        }
                        const bool top = j == 0;
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const int t = col0 + c;
                            const bool inBand = c >= cB && c <= cE;
                            const bool inR = c >= cRlo && c <= cRhi;
                            uint32_t &sw = c < 4 ? sreg0 : sreg1;
                            const int sh = 8 * (c & 3);
                            const uint32_t fresh = (uint32_t)prmt_sx(rlo[c], rhi[c], selj) & 0xffu;
                            if (inBand) sw = (sw & ~(0xffu << sh)) | (fresh << sh);
                            const int z0 = sx8(sw >> sh);
                            int lx = fx, lv = fv, lx2 = fx2;
                            int uu = top ? edge_diff(t, S) : ut[c];
                            int yy = top ? -S.qe : yt[c], yy2 = top ? -S.qe2 : y2t[c];
                            int d = 0;
                            cell<ARGMAX, RIGHT>(z0, lx, lv, lx2, uu, yy, yy2, d, S);
                            if (inR) ut[c] = uu, yt[c] = yy, y2t[c] = yy2;
                            fx = inR ? lx : -S.qe, fv = inR ? lv : -S.qe, fx2 = inR ? lx2 : -S.qe2;
                            const bool re = t == tm1 || top || c >= redge;
                            const int hn = r0 + c == 0 ? lv - S.qe_pre : (re && t > 0) ? Hf + uu : H[c] + lv;
                            if (inBand) {
                                H[c] = hn;
                                // end tracking straight into the pair's record (rare cells; the
                                // packed keys make the ">=" later-wins rule an unsigned max, and
                                // the strict earlier-wins rule one on the mirrored position)
                                const int pm = A.sse_st ? INT_MAX : 0;
                                if (re && t == tm1) atomicMax(&R->mte_key, end_key(hn, pm ^ j));
                                if (j == qm1) atomicMax(&R->mqe_key, end_key(hn, pm ^ t));
                                if (j == qm1 && t == tm1) R->score = hn, R->has_score = 1;
                            }
                            if (ARGMAX) {
                                const uint32_t dd = inR ? (uint32_t)d : 0u;
                                if (c < 4) w0 |= dd << (8 * c);
                                else w1 |= dd << (8 * (c - 4));
                            } else if (ST) {
                                const uint32_t bv = inR ? (uint32_t)(lv & 0xff) : 0u, bu = inR ? (uint32_t)(uu & 0xff) : 0u;
                                if (c < 4) w0 |= bv << (8 * c), w2 |= bu << (8 * c);
                                else w1 |= bv << (8 * (c - 4)), w3 |= bu << (8 * (c - 4));
                            }
                            Hf = H[c];
                        }
                    }
                    carry = pack3(fx, fv, fx2, qc);
                    Hcarry = Hf;
                }
                if (src_lane) ring[warp][k & 15][lane] = carry;
                if (store_tb && j >= jlo) {
                    uint8_t *dst = tbp + ((int64_t)(j - jlo + lane) * 32 + lane) * CB;
                    if (C == 8) {
                        if (ST) __stcs(reinterpret_cast<uint4 *>(dst), make_uint4(w0, w1, w2, w3));
                        else __stcs(reinterpret_cast<uint2 *>(dst), make_uint2(w0, w1));
                    } else {
                        if (ST) __stcs(reinterpret_cast<uint2 *>(dst), make_uint2(w0, w2));
                        else __stcs(reinterpret_cast<uint32_t *>(dst), w0);
                    }
                }
                if (lane == 31 && !last_strip && j >= jlo) bnd_me[j - jlo] = make_uint2(carry & 0xffffffu, (uint32_t)Hcarry);
            }
            if (lane == 31 && !last_strip) {
                const int jj = jstart + k - 31;
                if (jj >= jlo && jj <= jend && (((jj - jlo) & (PUB - 1)) == PUB - 1 || jj == jend)) {
                    if (jj == jend) bnd_me[jend - jlo + 1] = make_uint2(init_pack, (uint32_t)Hcarry);
                    // the release store orders this lane's boundary writes before the count
                    cuda::atomic_ref<int32_t, cuda::thread_scope_device> pw(*prog_me);
                    pw.store(jj == jend ? jj + 2 : jj + 1, cuda::memory_order_release);
                }
            }
            if (B > 16) __syncwarp();
        }
        if (failed) break;
    }
}

// ---- traceback --------------------------------------------------------------------

// CIGAR under construction, replicated in every lane of the walking warp: the open
// run stays in registers and lane 0 writes a run when the next op differs (the
// merge rule of ksw_push_cigar, minimap2/ksw2.h:144-154).
struct WarpCig {
    uint32_t *buf;
    int n;          // runs written
    uint32_t op;    // open run
    int len;        // 0 = no open run
    __device__ void push(uint32_t o, int l) {
        if (len > 0 && o == op) {
            len += l;
            return;
        }
        if (len > 0 && (threadIdx.x & 31) == 0) buf[n] = (uint32_t)len << 4 | op;
        if (len > 0) ++n;
        op = o, len = l;
    }
    __device__ int finish(bool reverse) {
        if (len > 0) {
            if ((threadIdx.x & 31) == 0) buf[n] = (uint32_t)len << 4 | op;
            ++n, len = 0;
        }
        __syncwarp();
        if (reverse) {
            const int lane = threadIdx.x & 31;
            for (int a = lane; a < n / 2; a += 32) {
                const uint32_t t = buf[a];
                buf[a] = buf[n - 1 - a], buf[n - 1 - a] = t;
            }
            __syncwarp();
        }
        return n;
    }
};

__device__ __forceinline__ int st_gap(int l, int o1, int e1, int o2, int e2) {
    if (l <= 0) return 0;
    const long long a = (long long)o1 + (long long)l * e1, b = (long long)o2 + (long long)l * e2;
    return (int)(a > b ? a : b);
}

struct BtArgs {
    const BandPairDev *pairs;
    int npair;
    const BandStripDev *strips;
    const uint8_t *tb;
    const BandRes *res;
    BandWalkState *walk;
    const uint8_t *qcodes, *tcodes;
    KswOut *out;
    uint32_t *cig;
    KswScore sc;
    int8_t mat[64];
    int m, flag, block;
};

// ksw_backtrack (minimap2/ksw2.h:160-192) over the strip layout with the band's
// off/off_end forcing, run in lockstep by a warp; stops when the walk ends or leaves the
// columns >= col_lo.
template <int NC, class Cache, class Load>
__device__ void band_walk(int &i, int &j, int &state, int col_lo, WarpCig &cg, Cache &cache, Load &load,
                          const Geom &g) {
    while (i >= 0 && j >= 0 && i >= col_lo) {
        const int r = i + j;
        int force = -1;
        if (i < (g.st0(r) & g.bmask)) force = 2;
        if (i > (g.en0(r) | 15)) force = 1;
        const uint32_t cellv = force < 0 ? cache.byte(i / NC, j, i % NC, load) : 0u;
        if (state == 0) state = cellv & 7;
        else if (!(cellv >> (state + 2) & 1)) state = 0;
        if (state == 0) state = cellv & 7;
        if (force >= 0) state = force;
        if (state == 0) cg.push(0, 1), --i, --j;
        else if (state == 1 || state == 3) cg.push(2, 1), --i;
        else cg.push(1, 1), --j;
    }
}

constexpr int FIN_WARPS = 4;

// Result record of one pair, then ksw_backtrack (minimap2/ksw2.h:160-192) with the
// off/off_end forcing of the band, or the Singletrack reconstruction
// (minimap2/ksw2_singletrack.cpp:63-176); one warp per pair walks with the tile cache.
template <bool ST, int NC>
__global__ void __launch_bounds__(32 * FIN_WARPS) ksw_band_finish_kernel(BtArgs A) {
    constexpr int WB = ST ? 2 * NC : NC;  // bytes per lane-word: NC columns (v then u for Singletrack)
    using Cache = TileCache<WB, 32, 64 / NC>;  // 32 rows x 64 columns
    __shared__ typename Cache::Word tiles[FIN_WARPS][2 * Cache::NW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pi = blockIdx.x * FIN_WARPS + warp;
    if (pi >= A.npair) return;
    const BandPairDev P = A.pairs[pi];
    const BandRes R = A.res[pi];
    const Geom g{P.qlen, P.tlen, P.w, P.qlen + P.tlen - 1, P.rb, ~(A.block - 1)};
    const int qlen = P.qlen, tlen = P.tlen, flag = A.flag;
    KswOut o;
    o.max = 0, o.max_q = -1, o.max_t = -1, o.reach_end = 0, o.stopped = 0, o.n_cigar = 0;
    o.score = R.has_score ? R.score : AW_NEG_INF;
    o.mqe = R.mqe_key ? (int)((uint32_t)(R.mqe_key >> 32) ^ 0x80000000u) : AW_NEG_INF;
    // ksw_extd2_singletrack_sse: positions stored mirrored (its strict ">"), and
    // mte_q = r - en with en rounded up to its 16-byte block (minimap2/ksw2_singletrack.cpp:583-586)
    const bool sse_st = (flag & AW_EZ_SINGLETRACK) && (flag & AW_EZ_SSE_SINGLETRACK);
    const int pm = sse_st ? INT_MAX : 0;
    o.mqe_t = R.mqe_key ? pm ^ (int)(uint32_t)R.mqe_key : -1;
    o.mte = R.mte_key ? (int)((uint32_t)(R.mte_key >> 32) ^ 0x80000000u) : AW_NEG_INF;
    o.mte_q = R.mte_key ? (pm ^ (int)(uint32_t)R.mte_key) - (sse_st ? ((tlen + 15) & ~15) - tlen : 0) : -1;
    o.zdropped = P.rb < g.nd ? 1 : 0;
    if (R.stopped) {
        // stopped at the deadline: no score and no traceback (ksw2_extd2_sse.c:136-139, :400-409)
        o.stopped = 1, o.score = AW_NEG_INF;
        if (lane == 0) {
            if (P.ckpt) A.walk[pi].done = 1;
            A.out[P.idx] = o;
        }
        return;
    }
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY);
    const BandStripDev *strips = A.strips + P.strip0;
    const uint8_t *tb = A.tb;
    Cache cache;
    cache.init(tiles[warp]);
    // the stored lane-word of column group gg (NC columns), row jj (zero outside the stored rows)
    auto load = [&](int gg, int jj) -> typename Cache::Word {
        typename Cache::Word z{};
        if (gg < 0 || jj < 0 || gg * NC >= tlen) return z;
        const int s = gg >> 5, L = gg & 31;
        const BandStripDev St = strips[s];
        if (jj < St.jlo || jj > St.jend) return z;
        const uint8_t *p = tb + St.tb_off + ((int64_t)(jj - St.jlo + L) * 32 + L) * WB;
        return __ldcs(reinterpret_cast<const typename Cache::Word *>(p));
    };
    auto stB = [&](int r) { return g.st0(r) & g.bmask; };
    auto en16 = [&](int r) { return (g.en0(r) & ~15) + 15; };
    WarpCig cg{A.cig + P.cig_off, 0, 0, 0};
    if (cigar && ST) {
        // ksw_extd2_singletrack_sse reconstructs whatever the EXTZ/SEMIGLOBAL flags
        // (minimap2/ksw2_singletrack.cpp:606-615)
        if (!o.zdropped && (sse_st || !(flag & (AW_EZ_EXTZ_ONLY | AW_EZ_SEMIGLOBAL_END)))) {
            const uint8_t *qs = A.qcodes + P.qoff, *ts = A.tcodes + P.toff;
            const int o1 = -A.sc.q, g1 = -A.sc.e, o2 = -A.sc.q2, g2 = -A.sc.e2;
            // track value (0 = v, 1 = u), the matrix-edge difference, or NEG_INF outside the stored band
            auto diff = [&](int part, int i, int j) -> int {
                if (i < 0 || j < 0) {
                    const int c = i < 0 ? j : i;
                    return st_gap(c + 1, o1, g1, o2, g2) - st_gap(c, o1, g1, o2, g2);
                }
                const int d = i + j;
                if (i < stB(d) || i > en16(d)) return AW_NEG_INF;
                return sx8(cache.byte(i / NC, j, (i % NC) + NC * part, load));
            };
            auto fin = [](int v) { return v > AW_NEG_INF / 2 && v < -AW_NEG_INF / 2; };
            bool in_m = true, valid = true;
            int i = tlen - 1, j = qlen - 1, l = 0, dd = 0, di = 0;
            while (i >= 0 && j >= 0) {
                const int dg = i + j;
                if (i < stB(dg)) { cg.push(1, 1); --j; in_m = true; continue; }
                if (i > en16(dg)) { cg.push(2, 1); --i; in_m = true; continue; }
                if (in_m) {
                    const int h = diff(0, i, j), v = diff(1, i, j - 1);
                    const int cost = A.mat[ts[i] * A.m + qs[j]];
                    if (fin(h) && fin(v) && (long long)h + v == cost) {
                        cg.push(0, 1);
                        --i, --j;
                    } else {
                        in_m = false, l = 0;
                        di = diff(0, i, j);
                        dd = diff(1, i, j);
                    }
                } else {
                    ++l;
                    if (l > i + 1 && l > j + 1) { valid = false; break; }
                    const int a1 = o1 + l * g1, a2 = o2 + l * g2, jn = j - l, id = i - l;
                    if (id >= -1 && (dd == a1 || dd == a2)) {
                        cg.push(2, l);
                        i = id, in_m = true;
                    } else if (jn >= -1 && (di == a1 || di == a2)) {
                        cg.push(1, l);
                        j = jn, in_m = true;
                    } else {
                        if (jn >= 0) {
                            const int Hh = diff(0, i, jn);
                            di = (fin(di) && fin(Hh)) ? di + Hh : AW_NEG_INF;
                        }
                        if (id >= 0) {
                            const int V = diff(1, id, j);
                            dd = (fin(dd) && fin(V)) ? dd + V : AW_NEG_INF;
                        }
                    }
                }
            }
            if (valid) {
                if (i >= 0) cg.push(2, i + 1);
                if (j >= 0) cg.push(1, j + 1);
                o.n_cigar = cg.finish(true);
            } else {
                o.n_cigar = 0;
            }
            if (o.n_cigar == 0) o.zdropped = 1;
        } else if (!o.zdropped) {
            o.zdropped = 1;
        }
    } else if (cigar) {
        int i0 = -1, j0 = -1;
        if (!o.zdropped && (flag & AW_EZ_SEMIGLOBAL_END)) {
            if (o.mqe > o.mte) o.score = o.mqe, i0 = o.mqe_t, j0 = qlen - 1;
            else o.score = o.mte, i0 = tlen - 1, j0 = o.mte_q;
        } else if (!o.zdropped && !(flag & AW_EZ_EXTZ_ONLY)) {
            i0 = tlen - 1, j0 = qlen - 1;
        }
        if (P.ckpt) {
            // traceback recomputed group by group (ksw_band_walk_kernel); start state only
            if (lane == 0) {
                BandWalkState w;
                w.i = i0, w.j = j0, w.state = 0, w.n = 0, w.op = 0, w.len = 0, w.pad = 0;
                w.done = (i0 >= 0 || j0 >= 0) ? 0 : 1;
                A.walk[pi] = w;
            }
        } else if (i0 >= 0 || j0 >= 0) {
            int i = i0, j = j0, state = 0;
            band_walk<NC>(i, j, state, 0, cg, cache, load, g);
            if (i >= 0) cg.push(2, i + 1);
            if (j >= 0) cg.push(1, j + 1);
            o.n_cigar = cg.finish(!(flag & AW_EZ_REV_CIGAR));
        }
    }
    if (lane == 0) A.out[P.idx] = o;
}

// One group of a recomputed pair per block (a round's groups): continue the ksw_backtrack
// walk through the group's freshly stored traceback until it leaves the group on the left
// (or ends); in the pair's first group, close the walk (the leading gap, the reversal, the
// CIGAR length).
template <int NC>
__global__ void __launch_bounds__(32) ksw_band_round_walk_kernel(BtArgs A, const BandGroupDev *groups) {
    using Cache = TileCache<NC, 32, 64 / NC>;
    __shared__ typename Cache::Word tiles[2 * Cache::NW];
    const BandGroupDev G = groups[blockIdx.x];
    const int slot = G.slot, col_lo = G.col_lo;
    BandWalkState w = A.walk[slot];
    if (w.done) return;
    const BandPairDev P = A.pairs[slot];
    if (A.res[slot].stopped) {
        // the group's recomputation stopped at the deadline: its traceback is incomplete
        if ((threadIdx.x & 31) == 0) {
            A.walk[slot].done = 1;
            A.out[P.idx].stopped = 1, A.out[P.idx].score = AW_NEG_INF, A.out[P.idx].n_cigar = 0;
        }
        return;
    }
    const Geom g{P.qlen, P.tlen, P.w, P.qlen + P.tlen - 1, P.rb, ~(A.block - 1)};
    const int tlen = P.tlen;
    const BandStripDev *strips = A.strips + P.strip0;
    const uint8_t *tb = A.tb;
    Cache cache;
    cache.init(tiles);
    auto load = [&](int gg, int jj) -> typename Cache::Word {
        typename Cache::Word z{};
        if (gg < 0 || jj < 0 || gg * NC >= tlen || gg * NC < col_lo) return z;
        const int s = gg >> 5, L = gg & 31;
        const BandStripDev St = strips[s];
        if (jj < St.jlo || jj > St.jend) return z;
        const uint8_t *p = tb + St.tb_off + ((int64_t)(jj - St.jlo + L) * 32 + L) * NC;
        return __ldcs(reinterpret_cast<const typename Cache::Word *>(p));
    };
    WarpCig cg{A.cig + P.cig_off, w.n, (uint32_t)w.op, w.len};
    int i = w.i, j = w.j, state = w.state;
    band_walk<NC>(i, j, state, col_lo, cg, cache, load, g);
    if (G.last) {
        if (i >= 0) cg.push(2, i + 1);
        if (j >= 0) cg.push(1, j + 1);
        const int n = cg.finish(!(A.flag & AW_EZ_REV_CIGAR));
        if ((threadIdx.x & 31) == 0) {
            A.out[P.idx].n_cigar = n;
            A.walk[slot].done = 1;
        }
        return;
    }
    if ((threadIdx.x & 31) == 0) {
        w.i = i, w.j = j, w.state = state, w.n = cg.n, w.op = (int)cg.op, w.len = cg.len;
        A.walk[slot] = w;
    }
}

// Progress counters of a round (one block per group): the group's strips start from zero, the
// strip on its left (not recomputed: its boundary column is stored from the first pass) counts
// as done.
__global__ void band_round_progress_kernel(int32_t *progress, const BandGroupDev *groups) {
    const BandGroupDev G = groups[blockIdx.x];
    for (int k = G.s_first + (int)threadIdx.x; k < G.s_end; k += blockDim.x) progress[PROG_STRIDE * k] = 0;
    if (threadIdx.x == 0 && G.left >= 0) progress[PROG_STRIDE * G.left] = INT_MAX / 2;
}

template <bool CIGAR, bool RIGHT, bool ST>
void *kernel_ptr() {
    return (void *)ksw_band_kernel<CIGAR, RIGHT, ST, 8>;
}

void *band_kernel_for(int flag, int block) {
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY), right = !!(flag & AW_EZ_RIGHT);
    const bool st = cigar && singletrack_tracks(flag, block);
    if (st) return kernel_ptr<true, false, true>();
    if (cigar && right) return kernel_ptr<true, true, false>();
    if (cigar) return kernel_ptr<true, false, false>();
    return kernel_ptr<false, false, false>();
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Device bytes of a pair's boundary columns (entries rounded as the wave packs them).
int64_t band_bnd_bytes(int64_t entries) { return (entries + 31) / 32 * 32 * (int64_t)sizeof(uint2); }

}  // namespace

int band_break(int qlen, int tlen, int w) {
    const int nd = qlen + tlen - 1;
    int rb = nd;
    if (w == 0 && nd > 1) rb = 1;
    // both conditions below are monotone in r (ksw2_extd2_sse.c:147-154: st > en)
    int lo = 0, hi = nd;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (mid - qlen + 1 > ((mid + w) >> 1)) hi = mid;
        else lo = mid + 1;
    }
    rb = std::min(rb, lo);
    lo = 0, hi = nd;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (((mid - w + 1) >> 1) > tlen - 1) hi = mid;
        else lo = mid + 1;
    }
    return std::min(rb, lo);
}

int64_t band_cells(int qlen, int tlen, int w) {
    if (w < 0) w = std::max(qlen, tlen);
    const int rb = band_break(qlen, tlen, w);
    int64_t total = 0;
    for (int r = 0; r < rb; ++r) {
        const int st = std::max(std::max(0, r - qlen + 1), (r - w + 1) >> 1);
        const int en = std::min(std::min(tlen - 1, r), (r + w) >> 1);
        total += en - st + 1;
    }
    return total;
}

int band_plan_build(BandPlan &bp, const std::vector<int32_t> &ids, const std::vector<int> &qlen,
                    const std::vector<int> &tlen, const std::vector<int> &w, const std::vector<KswPair> &pairs,
                    int flag, int block, int64_t tb_budget, int nc, std::vector<int32_t> *refused) {
    bp = BandPlan();
    bp.block = block;
    bp.nc = nc == 4 ? 4 : 8;
    const int SW = 32 * bp.nc;  // strip width
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY);
    const bool st = cigar && singletrack_tracks(flag, block);
    const int CB = st ? 2 * bp.nc : bp.nc;  // traceback bytes per lane-step
    const int B = block;
    struct PairGeo {
        int32_t id, ww, rb;
        int64_t tb, bnd;
        bool ckpt = false, refused = false, notb = false;
        std::vector<BandStripDev> strips;
        std::vector<int64_t> start;  // estimated start step of each strip
        std::vector<int64_t> stb;    // traceback bytes of each strip
    };
    std::vector<PairGeo> geo(ids.size());
    for (size_t a = 0; a < ids.size(); ++a) {
        PairGeo &G = geo[a];
        const int i = ids[a], ql = qlen[i], tl = tlen[i];
        const int ww = w[i] < 0 ? std::max(ql, tl) : std::min(w[i], std::max(ql, tl));
        G.id = i, G.ww = ww, G.rb = band_break(ql, tl, ww);
        const int nd = ql + tl - 1;
        const int nstrip = (int)ceil_div(tl, SW);
        G.tb = 0, G.bnd = 0;
        int64_t T = 0;
        int prev_js = 0;
        for (int s = 0; s < nstrip; ++s) {
            const int c0 = s * SW;
            BandStripDev sd;
            // rows the strip sweeps: from the first score-fill row of any of its columns
            // (fills reach 15 past en0, so no earlier than c0-w-31, and no row above -15)
            // to the last row where one of its columns is computed (stB <= t)
            sd.jstart = (int)std::max<int64_t>(-15, (int64_t)c0 - ww - 32);
            sd.jlo = std::max(0, sd.jstart);
            int64_t jend = -1;
            for (int tg = c0; tg < std::min(c0 + SW, tl); tg += B) {
                const int64_t X = (int64_t)tg + B - 1;
                const int64_t b = std::min<int64_t>(std::min<int64_t>(nd - 1, (int64_t)G.rb - 1),
                                                    std::min<int64_t>(X + ql - 1, 2 * X + ww));
                jend = std::max(jend, b - tg);
            }
            sd.jend = (int)std::min<int64_t>(jend, ql - 1);
            const int64_t rows = sd.jend >= sd.jlo ? (int64_t)sd.jend - sd.jlo + 1 : 0;
            sd.tb_off = G.tb;  // relative to the pair until the wave is packed
            sd.bnd_off = G.bnd;
            int64_t stb = 0;
            if (rows > 0) {
                if (cigar) stb = (rows + 31) * 32 * CB;
                G.tb += stb;
                G.bnd += rows + 1;
            }
            G.stb.push_back(stb);
            // estimated start: the left strip must have swept this strip's first rows
            T += (s == 0 ? 0 : std::max(0, sd.jstart - prev_js) + 64);
            prev_js = sd.jstart;
            G.strips.push_back(sd);
            G.start.push_back(T);
        }
        G.tb = (G.tb + 255) / 256 * 256;
        if (G.rb < nd) {
            // the band becomes empty before the end: the reference stops there with
            // zdropped = 1 and no traceback (ksw2_extd2_sse.c:151-154), so the DP runs without
            // storing one (the first pass of a recomputed pair, with nothing to recompute)
            G.ckpt = G.notb = true;
            G.tb = 0;
        }
    }
    // The budget is split once between the boundary-column arena and the traceback arena
    // (both are sized for their largest wave): the boundary columns get what the whole batch
    // needs, up to a third of the budget; the traceback arena the rest.  A wave's boundary
    // columns and its tracebacks stored in full must fit their arenas; the recompute rounds of
    // its recomputed pairs use the whole traceback arena after the wave's other walks.
    int64_t bnd_all = 0;
    for (const PairGeo &G : geo) bnd_all += band_bnd_bytes(G.bnd);
    const int64_t cap_bnd = std::min(bnd_all, tb_budget / 3);
    const int64_t cap_tb = std::max<int64_t>(tb_budget - cap_bnd, 1);
    const int64_t gres = cap_tb;
    for (PairGeo &G : geo) {
        if (G.notb) continue;
        // Singletrack pairs keep their whole two-track traceback: the reconstruction probes
        // arbitrarily far left in one gap search, so it cannot be split into strip groups.  A
        // pair whose traceback does not fit is refused like an allocation failure of the
        // reference (ksw2_extd2_avx.c:206-210: reset result, zdropped = 1).
        bool refuse = st && G.tb > cap_tb;
        if (!st && G.tb > cap_tb) {
            // Traceback beyond the budget: the first pass stores only the strips' boundary
            // columns; then the traceback is recomputed in groups of strips, from the last group
            // to the first, each from the stored column on its left, and the walk continues
            // through each group as it is recomputed.  The groups are cut per wave (below).
            for (int s = 0; s < (int)G.strips.size(); ++s) refuse |= G.stb[s] > cap_tb;
            if (!refuse) {
                G.ckpt = true;
                G.tb = 0;  // the first pass stores no traceback
            }
        }
        if (refuse) {
            if (!refused) return AW_E_NOMEM_INTERNAL;
            G.refused = true;
            refused->push_back(G.id);
        }
    }
    for (const PairGeo &G : geo) {
        if (G.refused) continue;
        bp.tb_total += G.tb;
        bp.cells += band_cells(qlen[G.id], tlen[G.id], G.ww);
    }
    // Pairs largest first into the fewest waves whose boundary columns and tracebacks stored in
    // full fit their arenas (LPT multiway fit), or one pair alone.
    std::vector<size_t> ord;
    for (size_t a = 0; a < ids.size(); ++a)
        if (!geo[a].refused) ord.push_back(a);
    std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
        const int64_t cx = (int64_t)qlen[geo[x].id] * geo[x].ww, cy = (int64_t)qlen[geo[y].id] * geo[y].ww;
        return cx != cy ? cx > cy : geo[x].id < geo[y].id;
    });
    std::vector<std::vector<size_t>> wv;
    std::vector<int64_t> wtb, wbnd;
    for (size_t a : ord) {
        const PairGeo &G = geo[a];
        const int64_t pb = band_bnd_bytes(G.bnd);
        int best = -1;
        for (size_t k = 0; k < wv.size(); ++k) {
            if (wtb[k] + G.tb <= cap_tb && wbnd[k] + pb <= cap_bnd &&
                (best < 0 || wbnd[k] * cap_tb + wtb[k] * cap_bnd < wbnd[best] * cap_tb + wtb[best] * cap_bnd))
                best = (int)k;
        }
        if (best < 0) {
            wv.emplace_back();
            wtb.push_back(0), wbnd.push_back(0);
            best = (int)wv.size() - 1;
        }
        wtb[best] += G.tb, wbnd[best] += pb;
        wv[best].push_back(a);
    }
    struct U {
        int64_t start;
        int slot, s;
    };
    auto by_start = [](const U &x, const U &y) {
        return x.start != y.start ? x.start < y.start : (x.slot != y.slot ? x.slot < y.slot : x.s < y.s);
    };
    for (size_t k = 0; k < wv.size(); ++k) {
        BandWave W;
        W.pair0 = (int)bp.pairs.size(), W.npair = (int)wv[k].size();
        W.unit0 = (int)bp.units.size(), W.strip0 = (int)bp.strips.size();
        int64_t tb = 0, bnd = 0;
        std::vector<U> us;
        std::vector<std::pair<int, size_t>> ck;  // (slot, geo index) of the recomputed pairs
        for (size_t a : wv[k]) {
            const PairGeo &G = geo[a];
            const KswPair &kp = pairs[G.id];
            BandPairDev pd;
            pd.qoff = kp.qoff, pd.toff = kp.toff, pd.cig_off = kp.cig_off;
            pd.qlen = kp.qlen, pd.tlen = kp.tlen, pd.w = G.ww, pd.rb = G.rb;
            pd.strip0 = (int)bp.strips.size();
            pd.nstrip = (int)G.strips.size();
            pd.idx = G.id, pd.ckpt = G.ckpt ? 1 : 0;
            const int slot = (int)bp.pairs.size();
            bp.pairs.push_back(pd);
            for (size_t s = 0; s < G.strips.size(); ++s) {
                BandStripDev sd = G.strips[s];
                if (!G.ckpt) sd.tb_off += tb;
                sd.bnd_off += bnd;
                bp.strips.push_back(sd);
                us.push_back(U{G.start[s], slot, (int)s});
            }
            if (G.ckpt && !G.notb) ck.push_back({slot, a});
            tb += G.tb;
            bnd += (G.bnd + 31) / 32 * 32;
        }
        // strips in estimated start order; a pair's strips keep their left-to-right order
        std::stable_sort(us.begin(), us.end(), by_start);
        for (const U &x : us) bp.units.push_back(make_int2(x.slot, x.s));
        W.nunit = (int)us.size();
        W.nstrip = (int)bp.strips.size() - W.strip0;
        W.tb_bytes = tb, W.bnd_entries = bnd;
        bp.tb_cap = std::max(bp.tb_cap, tb);
        bp.bnd_cap = std::max(bp.bnd_cap, bnd);
        // Recompute rounds: each recomputed pair gets a share of the round budget in proportion
        // to its whole traceback (so that all pairs need about as many rounds) and is cut into
        // groups of consecutive strips within it (at least one strip); round r recomputes the
        // r-th group from the right of every pair that has one, all together.
        W.round0 = (int)bp.rounds.size();
        std::vector<std::vector<std::pair<int, int>>> groups(ck.size());  // per pair: [s0, s1) right to left
        std::vector<std::vector<int64_t>> gtb(ck.size());
        double tb_all = 0;
        for (size_t c = 0; c < ck.size(); ++c)
            for (int64_t x : geo[ck[c].second].stb) tb_all += (double)x;
        size_t nround = 0;
        for (size_t c = 0; c < ck.size(); ++c) {
            const PairGeo &G = geo[ck[c].second];
            double tb_pair = 0;
            for (int64_t x : G.stb) tb_pair += (double)x;
            const int64_t share = std::max<int64_t>((int64_t)((double)gres * tb_pair / std::max(tb_all, 1.0)), 1);
            int s1 = (int)G.strips.size();
            while (s1 > 0) {
                int s0 = s1 - 1;
                int64_t acc = G.stb[s0];
                while (s0 > 0 && acc + G.stb[s0 - 1] <= share) acc += G.stb[--s0];
                groups[c].push_back({s0, s1});
                gtb[c].push_back(acc);
                s1 = s0;
            }
            nround = std::max(nround, groups[c].size());
        }
        for (size_t r = 0; r < nround; ++r) {
            BandRound R;
            R.group0 = (int)bp.groups.size(), R.unit0 = (int)bp.units.size(), R.nstrip = 0;
            int64_t off = 0;
            std::vector<U> ru;
            for (size_t c = 0; c < ck.size(); ++c) {
                if (r >= groups[c].size()) continue;
                const int slot = ck[c].first;
                const PairGeo &G = geo[ck[c].second];
                const BandPairDev &pd = bp.pairs[slot];
                const int s0 = groups[c][r].first, s1 = groups[c][r].second;
                BandGroupDev gd;
                gd.slot = slot, gd.s_first = pd.strip0 + s0, gd.s_end = pd.strip0 + s1;
                gd.left = s0 > 0 ? pd.strip0 + s0 - 1 : -1;
                gd.col_lo = s0 * SW;
                gd.last = r + 1 == groups[c].size() ? 1 : 0;
                gd.pad0 = gd.pad1 = 0;
                bp.groups.push_back(gd);
                int64_t o = off;
                for (int s = s0; s < s1; ++s) {
                    bp.strips[pd.strip0 + s].tb_off = o;  // this round's arena
                    o += G.stb[s];
                    ru.push_back(U{G.start[s] - G.start[s0], slot, s});
                }
                off += gtb[c][r];
                R.nstrip += s1 - s0;
            }
            std::stable_sort(ru.begin(), ru.end(), by_start);
            for (const U &x : ru) bp.units.push_back(make_int2(x.slot, x.s));
            R.ngroup = (int)bp.groups.size() - R.group0;
            R.nunit = (int)ru.size();
            R.tb_bytes = off;
            bp.tb_cap = std::max(bp.tb_cap, off);
            bp.rounds.push_back(R);
        }
        W.nround = (int)bp.rounds.size() - W.round0;
        bp.waves.push_back(W);
    }
    return 0;
}

int band_occupancy(int flag) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, band_kernel_for(flag, 64), 256, 0) != cudaSuccess) return 1;
    return std::max(nb, 1);
}

cudaError_t band_launch_units(const BandPlan &bp, const BandArgs &a, int flag, int ctas, cudaStream_t st);

cudaError_t band_launch_dp(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                           const uint8_t *tcodes, const KswScore &S, int flag, int ctas, cudaStream_t st) {
    const BandWave &W = bp.waves[k];
    cudaError_t e;
    if ((e = cudaMemsetAsync(D.progress + (size_t)PROG_STRIDE * W.strip0, 0,
                             sizeof(int32_t) * PROG_STRIDE * std::max(W.nstrip, 1), st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(D.res + W.pair0, 0, sizeof(BandRes) * std::max(W.npair, 1), st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(D.queue + 64 * k, 0, sizeof(int32_t), st)) != cudaSuccess) return e;
    BandArgs a;
    a.qcodes = qcodes, a.tcodes = tcodes;
    a.pairs = D.pairs, a.strips = D.strips, a.units = D.units + W.unit0;
    a.n_units = W.nunit;
    a.queue = D.queue + 64 * k, a.progress = D.progress, a.error = D.error;
    a.tb = D.tb, a.bnd = D.bnd, a.res = D.res;
    a.sc = S;
    a.block = bp.block;
    a.generic = (flag & AW_EZ_GENERIC_SC) ? 1 : 0;
    a.sse_st = (flag & AW_EZ_SINGLETRACK) && (flag & AW_EZ_SSE_SINGLETRACK) ? 1 : 0;
    a.store_ckpt = 0;
    a.deadline = D.deadline;
    a.walk = nullptr;
    return band_launch_units(bp, a, flag, ctas, st);
}

cudaError_t band_launch_units(const BandPlan &bp, const BandArgs &a, int flag, int ctas, cudaStream_t st) {
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY), right = !!(flag & AW_EZ_RIGHT);
    const bool stk = cigar && singletrack_tracks(flag, bp.block);
    const int grid = std::max(1, std::min(ctas, (a.n_units + 7) / 8));
#define AW_BAND_LAUNCH(NCV)                                                                   \
    if (stk) ksw_band_kernel<true, false, true, NCV><<<grid, 256, 0, st>>>(a);               \
    else if (cigar && right) ksw_band_kernel<true, true, false, NCV><<<grid, 256, 0, st>>>(a); \
    else if (cigar) ksw_band_kernel<true, false, false, NCV><<<grid, 256, 0, st>>>(a);        \
    else ksw_band_kernel<false, false, false, NCV><<<grid, 256, 0, st>>>(a);
    if (bp.nc == 4) {
        AW_BAND_LAUNCH(4)
    } else {
        AW_BAND_LAUNCH(8)
    }
#undef AW_BAND_LAUNCH
    return cudaGetLastError();
}

cudaError_t band_launch_finish(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                               const uint8_t *tcodes, const KswScore &S, int flag, KswOut *out, uint32_t *cig,
                               const int8_t *mat, int m, cudaStream_t st) {
    const BandWave &W = bp.waves[k];
    BtArgs b;
    b.pairs = D.pairs + W.pair0, b.npair = W.npair, b.strips = D.strips, b.tb = D.tb, b.res = D.res + W.pair0;
    b.walk = D.walk + W.pair0;
    b.qcodes = qcodes, b.tcodes = tcodes, b.out = out, b.cig = cig, b.sc = S;
    memset(b.mat, 0, sizeof(b.mat));
    memcpy(b.mat, mat, (size_t)m * m);
    b.m = m, b.flag = flag, b.block = bp.block;
    const int grid = (W.npair + FIN_WARPS - 1) / FIN_WARPS;
    const bool stk = singletrack_tracks(flag, b.block) && !(flag & AW_EZ_SCORE_ONLY);
    if (bp.nc == 4) {
        if (stk) ksw_band_finish_kernel<true, 4><<<grid, 32 * FIN_WARPS, 0, st>>>(b);
        else ksw_band_finish_kernel<false, 4><<<grid, 32 * FIN_WARPS, 0, st>>>(b);
    } else {
        if (stk) ksw_band_finish_kernel<true, 8><<<grid, 32 * FIN_WARPS, 0, st>>>(b);
        else ksw_band_finish_kernel<false, 8><<<grid, 32 * FIN_WARPS, 0, st>>>(b);
    }
    return cudaGetLastError();
}

cudaError_t band_launch_groups(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                               const uint8_t *tcodes, const KswScore &S, int flag, KswOut *out, uint32_t *cig,
                               const int8_t *mat, int m, int ctas, cudaStream_t st) {
    const BandWave &W = bp.waves[k];
    cudaError_t e;
    BtArgs b;
    b.pairs = D.pairs, b.npair = (int)bp.pairs.size(), b.strips = D.strips, b.tb = D.tb, b.res = D.res;
    b.walk = D.walk;
    b.qcodes = qcodes, b.tcodes = tcodes, b.out = out, b.cig = cig, b.sc = S;
    memset(b.mat, 0, sizeof(b.mat));
    memcpy(b.mat, mat, (size_t)m * m);
    b.m = m, b.flag = flag, b.block = bp.block;
    for (int ri = W.round0; ri < W.round0 + W.nround; ++ri) {
        const BandRound &R = bp.rounds[ri];
        const BandGroupDev *gd = D.groups + R.group0;
        band_round_progress_kernel<<<R.ngroup, 256, 0, st>>>(D.progress, gd);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        // this round's counter of the work queue: the wave's slot, reused per round
        if ((e = cudaMemsetAsync(D.queue + 64 * k, 0, sizeof(int32_t), st)) != cudaSuccess) return e;
        BandArgs a;
        a.qcodes = qcodes, a.tcodes = tcodes;
        a.pairs = D.pairs, a.strips = D.strips, a.units = D.units + R.unit0;
        a.n_units = R.nunit;
        a.queue = D.queue + 64 * k, a.progress = D.progress, a.error = D.error;
        a.tb = D.tb, a.bnd = D.bnd, a.res = D.res;
        a.sc = S;
        a.block = bp.block;
        a.generic = (flag & AW_EZ_GENERIC_SC) ? 1 : 0;
        a.sse_st = (flag & AW_EZ_SINGLETRACK) && (flag & AW_EZ_SSE_SINGLETRACK) ? 1 : 0;
        a.store_ckpt = 1;
        a.deadline = D.deadline;
        a.walk = D.walk;
        if ((e = band_launch_units(bp, a, flag, ctas, st)) != cudaSuccess) return e;
        if (bp.nc == 4) ksw_band_round_walk_kernel<4><<<R.ngroup, 32, 0, st>>>(b, gd);
        else ksw_band_round_walk_kernel<8><<<R.ngroup, 32, 0, st>>>(b, gd);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace aw
