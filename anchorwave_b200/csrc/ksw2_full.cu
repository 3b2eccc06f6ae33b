// KSW2 extd2, full-matrix form (w < 0 or w >= max(qlen, tlen)), on sm_100a.
//
// Same recurrence as minimap2/ksw2_extd2_sse.c:43-71 + :237-330 (difference-
// encoded u, v, x, y, x2, y2 cells; state byte d with the 3-bit argmax and the
// four continuation bits).  In full mode every cell the recurrence reads is a real
// matrix cell or a matrix edge, so the SIMD padding lanes of the reference never
// influence the result and are not computed here.  The host only routes parameter
// sets to this kernel whose int8 intermediates provably cannot wrap
// (ksw2_api.cu: full_path_ok).
//
// Two cells per instruction.  Every register holds two 16-bit fields, each a cell
// value stored as 16*value + bias; the two fields are cells of two different rows
// (below), so a cell is DPX SIMD (vimax3 / viaddmin .s16x2, vmax / vmin .s16x2) plus
// 32-bit adds whose per-field results stay inside [0, 65536), which the biases
// guarantee, so no carry crosses from one field into the other.  The low 4 bits of a
// field are free: the five candidates of the max carry a priority tag there, so one
// max yields both z and the arg-max under the reference's tie rule (left-aligned: the
// first candidate wins a tie, ksw2_extd2_sse.c:244-251; right-aligned: the last,
// :291-298).
//
// Work decomposition (one pair per group of W warps):
//   * target columns are cut into strips of 512 (32 lanes x 16 columns); lane L owns
//     columns 16L..16L+7 in its low fields and 16L+8..16L+15 in its high fields;
//   * a warp sweeps the query rows of its strip with a skew of two steps per lane and
//     one step between the halves: at step k lane L computes row k-2L in its low fields
//     and row k-2L-1 in its high fields, so the (x, v, x2) of its low column 7 feed its
//     high column 8 at the next step, and its high column 15 reaches lane L+1 by one
//     __shfl_up per step, together with the query code of that row;
//   * strip s+1 takes its left edge (column 512(s+1)-1 of strip s) from a global
//     boundary buffer that strip s fills row by row; with W > 1 the W warps of a group
//     run consecutive strips concurrently, the consumer warp polling the producer's
//     published row count in shared memory (bounded);
//   * the traceback bytes of a step go to HBM as one coalesced 512-byte store per warp
//     (16 bytes per lane), with evict-first policy (they are read back along one path);
//   * H is not carried per cell: the last row's H (mqe, the score) is a prefix sum of
//     the last row's u along the strip after the sweep, and the last column's H (mte)
//     is accumulated by the lane that owns that column.
// Pairs are pulled from a device work queue (atomicAdd on a head counter) in the
// host-provided order (largest first), so one persistent launch serves a whole batch
// of uneven pairs.
#include "aw_internal.h"
#include "tb_walk.cuh"
#include <cuda/atomic>
#include <atomic>

namespace aw {

namespace {

constexpr int MAX_GROUP_WARPS = 32;
constexpr unsigned FULLMASK = 0xffffffffu;

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

// Difference along a matrix edge for edge cell index r (ksw2_extd2_sse.c:167,171).
__device__ __forceinline__ int edge_diff(int r, const KswScore &S) {
    return r == 0 ? -S.qe : r < S.long_thres ? -S.e : r == S.long_thres ? S.long_diff : -S.e2;
}

// H(t, -1) (= H(-1, t)): sum of edge_diff(0..t), the score of a leading gap of length
// t+1, offset as the reference's H[0] = v[0] - qe with qe taken before the swap.
__device__ __forceinline__ int htop(int t, const KswScore &S) {
    const int L = S.long_thres;
    int A = min(t, L - 1);
    A = A < 0 ? 0 : A;
    const int eq = (L >= 1 && L <= t) ? 1 : 0;
    const int B = t - A - eq;
    // the reference seeds H[0] with the pre-swap q+e, which shifts every H equally
    return -S.qe_pre - A * S.e + eq * S.long_diff - B * S.e2;
}

__device__ __forceinline__ void group_sync(int g, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(nthreads) : "memory");
}

// ---- packed cell fields ------------------------------------------------------------
// Every field holds 16*value + FB; x, y, x2, y2 carry their candidate's priority tag on
// top (so x + v is already the tagged candidate a), and the score carries 2*FB + its tag.
// With the magnitude bound of full_path_ok (|u|, |v|, |x|, ... <= 300, and the bounded
// excursions of masked-off fields within one step) every 32-bit add below keeps each field
// inside [0, 65536) and every value a DPX op compares for a live field inside [0, 32768).
// The adds are 2-input multiply-adds by a runtime one (or minus one), so they issue on the
// FMA pipe and leave the ALU pipe to the max/min/permute work.
constexpr int FB = 12288;
// A constant in both fields: for 32-bit adds (c * 65537, so that a negative c borrows
// exactly what the field sum carries back) and for SIMD operands (each field = c).
__host__ __device__ constexpr uint32_t add2(int c) { return (uint32_t)c * 0x10001u; }
__host__ __device__ constexpr uint32_t rep2(int c) { return ((uint32_t)c & 0xffffu) * 0x10001u; }

// Priority tags of the candidates s, a, b, a2, b2 (the larger tag wins a tie of values),
// and the XOR that turns the winning tag into the reference's state code d (0 = s, 1 = a,
// 2 = b, 3 = a2, 4 = b2).  Score-only sweeps need no arg-max: no tags.
template <bool CIGAR, bool RIGHT>
struct Tags {
    static constexpr int s = !CIGAR ? 0 : RIGHT ? 0 : 7;
    static constexpr int a = !CIGAR ? 0 : RIGHT ? 1 : 6;
    static constexpr int b = !CIGAR ? 0 : RIGHT ? 2 : 5;
    static constexpr int a2 = !CIGAR ? 0 : RIGHT ? 3 : 4;
    static constexpr int b2 = !CIGAR ? 0 : RIGHT ? 4 : 3;
    static constexpr uint32_t dx = (CIGAR && !RIGHT) ? 0x00070007u : 0u;
};

// Per-launch packed constants of the cell.
struct CellK {
    uint32_t ke, ke2;               // Ze = Z + ke: W = candidate - Ze = 16 (cand - z - e) + FB + tag
    uint32_t kxa, kxb, kxa2, kxb2;  // x' = max(W, kx): the field of -(q+e) (-(q2+e2)) with the tag (SIMD)
    uint32_t ca, cb, ca2, cb2;      // continuation: relu(min(W + c, 8 or 16))       (SIMD)
    uint32_t mch;                   // z = min(z, mch)                                (SIMD)
    uint32_t one, neg1;             // runtime 1 and -1 of the multiply-adds
};

template <bool CIGAR, bool RIGHT>
__device__ __forceinline__ CellK make_cellk(const KswScore &S, uint32_t one) {
    using T = Tags<CIGAR, RIGHT>;
    CellK K;
    K.ke = add2(16 * S.e - FB), K.ke2 = add2(16 * S.e2 - FB);
    const int xa = FB - 16 * S.qe + T::a, xb = FB - 16 * S.qe + T::b;
    const int xa2 = FB - 16 * S.qe2 + T::a2, xb2 = FB - 16 * S.qe2 + T::b2;
    K.kxa = rep2(xa), K.kxb = rep2(xb), K.kxa2 = rep2(xa2), K.kxb2 = rep2(xb2);
    // left-aligned: a - z + q > 0 (ksw2_extd2_sse.c:268-271) <=> W - kx >= 16;
    // right-aligned: >= 0 (:315-318) <=> W - kx >= 0.  The a bit is 8, the others 16
    // (scaled to 32 and 64 when they are added to the state byte).
    K.ca = rep2((RIGHT ? 8 : -8) - xa), K.cb = rep2((RIGHT ? 16 : 0) - xb);
    K.ca2 = rep2((RIGHT ? 16 : 0) - xa2), K.cb2 = rep2((RIGHT ? 16 : 0) - xb2);
    K.mch = rep2(16 * S.mch + 2 * FB);
    K.one = one, K.neg1 = 0u - one;
    return K;
}

// Two cells, one per field.  In: sc (tagged score), X/V/X2 from the left column, U/Y/Y2
// the column state from the row above.  Out: X/V/X2 for the next column, U/Y/Y2 for
// the next row, D the two state bytes (one per field).
template <bool CIGAR, bool RIGHT>
__device__ __forceinline__ void cell2(uint32_t sc, uint32_t &X, uint32_t &V, uint32_t &X2, uint32_t &U,
                                      uint32_t &Y, uint32_t &Y2, uint32_t &D, const CellK &K) {
    // a = x + v, b = y + u, a2 = x2 + v, b2 = y2 + u (ksw2_extd2_sse.c:240-243), tagged
    const uint32_t A = X * K.one + V, Bv = Y * K.one + U, A2 = X2 * K.one + V, B2 = Y2 * K.one + U;
    uint32_t Z = __vimax3_s16x2(__vimax3_s16x2(sc, Bv, B2), A, A2);
    if (CIGAR) {
        D = (Z & 0x000f000fu) ^ Tags<CIGAR, RIGHT>::dx;
        Z &= 0xfff0fff0u;
    }
    Z = __vmins2(Z, K.mch);  // ksw2_extd2_sse.c:252
    const uint32_t Un = V * K.neg1 + Z, Vn = U * K.neg1 + Z;
    const uint32_t Ze = Z * K.one + K.ke, Ze2 = Z * K.one + K.ke2;
    const uint32_t Wa = Ze * K.neg1 + A, Wb = Ze * K.neg1 + Bv, Wa2 = Ze2 * K.neg1 + A2, Wb2 = Ze2 * K.neg1 + B2;
    X = __vmaxs2(Wa, K.kxa);
    Y = __vmaxs2(Wb, K.kxb);
    X2 = __vmaxs2(Wa2, K.kxa2);
    Y2 = __vmaxs2(Wb2, K.kxb2);
    if (CIGAR) {
        D = __viaddmin_s16x2_relu(Wa, K.ca, 0x00080008u) * K.one + D;
        D = __viaddmin_s16x2_relu(Wb, K.cb, 0x00100010u) * K.one + D;
        D = __viaddmin_s16x2_relu(Wa2, K.ca2, 0x00100010u) * 2u + D;
        D = __viaddmin_s16x2_relu(Wb2, K.cb2, 0x00100010u) * 4u + D;
    }
    U = Un;
    V = Vn;
}

__device__ __forceinline__ int fld(uint32_t w, int f) { return f ? (int)(w >> 16) : (int)(w & 0xffffu); }

// Lexicographic (value, position) maximum: later positions win ties, the
// ">=" end-tracking rule of ksw2_extd2_sse.c:369-372.
__device__ __forceinline__ void best_merge(int &v, int &p, int ov, int op) {
    if (ov > v || (ov == v && op > p)) v = ov, p = op;
}

// Score profile of a lane: for each query code q (0..7) the 16 tagged score fields of the
// lane's columns, 256 B per lane in shared memory, read back by the same lane only.  The
// low columns (0..7) and the high columns (8..15) are 16 B each; lanes with bit 2 set store
// them swapped, so the 8 lanes of a quarter-warp load 16 B each from distinct banks.
constexpr int PROF_LANE = 32;                 // bytes per lane and code
constexpr int PROF_CODE = 32 * PROF_LANE;     // bytes per code (one warp)
constexpr int PROF_WARP = 8 * PROF_CODE;      // bytes per warp

// State of one warp's sweep over one strip.
struct Sweep {
    uint32_t U[8], Y[8], Y2[8];  // column state, column pair c = (col0 + c, col0 + 8 + c)
    uint32_t X, V, X2;           // values flowing right; after a step: the outputs of column pair 7
    uint32_t qlo, qhi;           // query codes of the rows of the low / high fields at the last step
    uint32_t vcap;               // last strip: v of the pair's last column at the last step
};

__device__ __forceinline__ uint32_t u4w(const uint4 &v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }

// One step of a warp: rows jlo = k - 2*lane (low fields) and jlo - 1 (high fields).
// r0/r1: the left values of the low fields ([x, v] and [x2, query code]); the high fields
// take the low fields' column 7 of the previous step.  MASKED: some field of the warp is
// outside [0, qlen): those fields start from safe left values and keep their column
// state.  LAST: capture v of column pair cc.
template <bool CIGAR, bool RIGHT, bool MASKED, bool LAST>
__device__ __forceinline__ void sweep_step(Sweep &w, uint32_t r0, uint32_t r1, uint32_t M, int cc, const CellK &K,
                                           const uint8_t *prof_lo, const uint8_t *prof_hi, uint8_t *tbdst) {
    uint32_t X = prmt(r0, w.X, 0x5410), V = prmt(r0, w.V, 0x5432), X2 = prmt(r1, w.X2, 0x5410);
    if (MASKED) {
        X = (X & M) | (K.kxa & ~M);
        V = (V & M) | (rep2(FB) & ~M);
        X2 = (X2 & M) | (K.kxa2 & ~M);
    }
    const uint32_t qlo = r1 >> 16, qhi = w.qlo;
    const uint4 slo = *reinterpret_cast<const uint4 *>(prof_lo + qlo * PROF_CODE);
    const uint4 shi = *reinterpret_cast<const uint4 *>(prof_hi + qhi * PROF_CODE);
    uint32_t D[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t sc = prmt(u4w(slo, c >> 1), u4w(shi, c >> 1), (c & 1) ? 0x7632 : 0x5410);
        uint32_t u = w.U[c], y = w.Y[c], y2 = w.Y2[c];
        cell2<CIGAR, RIGHT>(sc, X, V, X2, u, y, y2, D[c], K);
        if (MASKED) {
            w.U[c] = (u & M) | (w.U[c] & ~M);
            w.Y[c] = (y & M) | (w.Y[c] & ~M);
            w.Y2[c] = (y2 & M) | (w.Y2[c] & ~M);
        } else {
            w.U[c] = u, w.Y[c] = y, w.Y2[c] = y2;
        }
        if (LAST && c == cc) w.vcap = V;
    }
    w.X = X, w.V = V, w.X2 = X2;
    w.qlo = qlo, w.qhi = qhi;
    if (CIGAR) {
        const uint32_t e01 = D[0] + D[1] * 256u, e23 = D[2] + D[3] * 256u;
        const uint32_t e45 = D[4] + D[5] * 256u, e67 = D[6] + D[7] * 256u;
        const uint4 v = make_uint4(prmt(e01, e23, 0x5410), prmt(e45, e67, 0x5410), prmt(e01, e23, 0x7632),
                                   prmt(e45, e67, 0x7632));
        __stcs(reinterpret_cast<uint4 *>(tbdst), v);
    }
}

// Per-strip context shared by the steps.
struct StripCtx {
    int qlen, lane, s, nstrip, c_lane, c_fld, c_cc;
    uint2 *bnd;                 // this pair's boundary columns
    int64_t bstride;            // entries per strip
    int *prog;                  // this warp's published progress (shared memory)
    int pstride;
    const uint8_t *prof_lo, *prof_hi;
    uint8_t *tb;                // this lane's traceback word of step 0 of the strip
    bool bnd_writer;            // lane 31 of a strip with a right neighbour
};

// Steps [k0, k1) of a strip; bx/by: lane i holds the left values of lane 0 for row k0 + i.
template <bool CIGAR, bool RIGHT, bool MASKED, bool LAST>
__device__ __forceinline__ void sweep_chunk(Sweep &w, const StripCtx &C, int k0, int k1, uint32_t bx, uint32_t by,
                                            const CellK &K, int &hm16, int &mte16, int &mte_q) {
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        const uint32_t w0 = prmt(w.X, w.V, 0x7632), w1 = prmt(w.X2, w.qhi, 0x5432);
        uint32_t r0 = __shfl_up_sync(FULLMASK, w0, 1), r1 = __shfl_up_sync(FULLMASK, w1, 1);
        const uint32_t b0 = __shfl_sync(FULLMASK, bx, k - k0), b1 = __shfl_sync(FULLMASK, by, k - k0);
        if (C.lane == 0) r0 = b0, r1 = b1;
        const int jlo = k - 2 * C.lane;
        uint32_t M = 0xffffffffu;
        if (MASKED)
            M = ((unsigned)jlo < (unsigned)C.qlen ? 0x0000ffffu : 0u) |
                ((unsigned)(jlo - 1) < (unsigned)C.qlen ? 0xffff0000u : 0u);
        uint8_t *tbdst = CIGAR ? C.tb + (int64_t)k * (32 * 16) : nullptr;
        sweep_step<CIGAR, RIGHT, MASKED, LAST>(w, r0, r1, M, C.c_cc, K, C.prof_lo, C.prof_hi, tbdst);
        if (LAST && C.lane == C.c_lane) {
            const int row = jlo - C.c_fld;
            if ((unsigned)row < (unsigned)C.qlen) {
                hm16 += fld(w.vcap, C.c_fld) - FB;
                if (hm16 >= mte16) mte16 = hm16, mte_q = row;
            }
        }
        if (C.bnd_writer) {
            const int jj = k - KSW_LAG;  // row of the high fields of lane 31
            if ((unsigned)jj < (unsigned)C.qlen) {
                C.bnd[(int64_t)C.s * C.bstride + jj] = make_uint2(prmt(w.X, w.V, 0x7632), w.X2 >> 16);
                if ((jj & 31) == 31 || jj == C.qlen - 1) {
                    // the consumer reads these rows from L2 (ld.cg), so they must be
                    // visible at device scope before the row count is published
                    __threadfence();
                    cuda::atomic_ref<int, cuda::thread_scope_block> pw(*C.prog);
                    pw.store(C.s * C.pstride + jj + 1, cuda::memory_order_release);
                }
            }
        }
    }
}

template <bool CIGAR, bool RIGHT, bool LAST>
__device__ __forceinline__ void sweep_range(Sweep &w, const StripCtx &C, int k0, int k1, uint32_t bx, uint32_t by,
                                            const CellK &K, int &hm16, int &mte16, int &mte_q) {
    // every field of every lane is inside [0, qlen) for k in [KSW_LAG, qlen)
    const int f0 = max(k0, KSW_LAG), f1 = min(k1, C.qlen);
    if (f0 >= f1) {
        sweep_chunk<CIGAR, RIGHT, true, LAST>(w, C, k0, k1, bx, by, K, hm16, mte16, mte_q);
        return;
    }
    // the chunk's sub-ranges keep the lane-0 words of row k0 + i in lane i
    if (k0 < f0) sweep_chunk<CIGAR, RIGHT, true, LAST>(w, C, k0, f0, bx, by, K, hm16, mte16, mte_q);
    sweep_chunk<CIGAR, RIGHT, false, LAST>(w, C, f0, f1, __shfl_down_sync(FULLMASK, bx, f0 - k0),
                                           __shfl_down_sync(FULLMASK, by, f0 - k0), K, hm16, mte16, mte_q);
    if (f1 < k1)
        sweep_chunk<CIGAR, RIGHT, true, LAST>(w, C, f1, k1, __shfl_down_sync(FULLMASK, bx, f1 - k0),
                                              __shfl_down_sync(FULLMASK, by, f1 - k0), K, hm16, mte16, mte_q);
}

template <bool CIGAR, bool RIGHT, int W>
__global__ void __launch_bounds__(256, 2) ksw_full_kernel(KswFullArgs A) {
    extern __shared__ __align__(16) uint8_t prof_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = warp / W;
    const int wg = warp % W;
    const KswScore &S = A.sc;
    const CellK K = make_cellk<CIGAR, RIGHT>(S, A.one);
    __shared__ int s_pair[MAX_GROUP_WARPS];
    __shared__ int s_prog[MAX_GROUP_WARPS];  // progress published, per warp (monotone per pair)
    __shared__ int s_red[MAX_GROUP_WARPS][5];
    __shared__ int s_stop[MAX_GROUP_WARPS];  // the group's pair passed the deadline
    int *prog = s_prog + g * W;
    volatile int *stop_flag = s_stop + g;
    uint8_t *prof = prof_smem + warp * PROF_WARP + lane * PROF_LANE;
    const int sw = (lane >> 2) & 1;
    using T = Tags<CIGAR, RIGHT>;

    for (;;) {
        group_sync(g, W * 32);
        if (wg == 0 && lane == 0) {
            s_pair[g] = atomicAdd(A.queue, 1);
            for (int i = 0; i < W; ++i) prog[i] = -1;
            *stop_flag = 0;
        }
        group_sync(g, W * 32);
        const int pi = s_pair[g];
        if (pi >= A.n) break;
        const int idx = A.order[pi];
        const KswPair P = A.pairs[idx];
        const int qlen = P.qlen, tlen = P.tlen;
        const uint8_t *qs = A.qcodes + P.qoff;
        const uint8_t *ts = A.tcodes + P.toff;
        const int nstrip = (tlen + KSW_STRIP - 1) / KSW_STRIP;
        const int tl1 = tlen - 1;
        StripCtx C;
        C.qlen = qlen, C.lane = lane, C.nstrip = nstrip;
        // boundary column of strip s: rows at [s * (qlen + 1), +qlen), its last-row H after them
        C.bnd = reinterpret_cast<uint2 *>(A.bnd + P.bnd_off);
        C.bstride = qlen + 1;
        C.prog = prog + wg;
        // progress of a warp: strip * pstride + (rows published, then +1 for the last-row H)
        C.pstride = qlen + 2;
        C.prof_lo = prof + 16 * sw, C.prof_hi = prof + 16 * (1 - sw);
        // the pair's last column: owning lane, field and column pair (in the last strip)
        C.c_lane = (tl1 % KSW_STRIP) >> 4, C.c_fld = (tl1 >> 3) & 1, C.c_cc = tl1 & 7;
        const int64_t stride_k = qlen + KSW_LAG;
        int mqe16 = INT_MIN, mqe_t = -1, mte16 = INT_MIN, mte_q = -1, score16 = INT_MIN;
        bool stopped = false;

        for (int s = wg; s < nstrip && !stopped; s += W) {
            const int col0 = s * KSW_STRIP + lane * 16;
            const bool last = s == nstrip - 1;
            C.s = s;
            C.bnd_writer = lane == 31 && s + 1 < nstrip;
            C.tb = CIGAR ? A.tb + P.tb_off + ((int64_t)s * stride_k * 32 + lane) * 16 : nullptr;
            // score profile of the lane's 16 columns for query codes 0..7
            {
                uint32_t tlo[16], thi[16];
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int col = col0 + c;
                    const int tc = col < tlen ? (ts[col] & 7) : 0;
                    tlo[c] = S.tab_lo[tc], thi[c] = S.tab_hi[tc];
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    uint32_t wd[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int sa = (int)(int8_t)(uint8_t)(((q < 4 ? tlo[2 * i] : thi[2 * i]) >> (8 * (q & 3))) & 0xff);
                        const int sb =
                            (int)(int8_t)(uint8_t)(((q < 4 ? tlo[2 * i + 1] : thi[2 * i + 1]) >> (8 * (q & 3))) & 0xff);
                        wd[i] = (uint32_t)(16 * sa + T::s + 2 * FB) | ((uint32_t)(16 * sb + T::s + 2 * FB) << 16);
                    }
                    *reinterpret_cast<uint4 *>(prof + q * PROF_CODE + 16 * sw) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
                    *reinterpret_cast<uint4 *>(prof + q * PROF_CODE + 16 * (1 - sw)) =
                        make_uint4(wd[4], wd[5], wd[6], wd[7]);
                }
            }
            Sweep w;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                w.U[c] = (uint32_t)(16 * edge_diff(col0 + c, S) + FB) |
                         ((uint32_t)(16 * edge_diff(col0 + 8 + c, S) + FB) << 16);
                w.Y[c] = K.kxb;
                w.Y2[c] = K.kxb2;
            }
            w.X = K.kxa, w.V = rep2(FB), w.X2 = K.kxa2;
            w.qlo = 0, w.qhi = 0, w.vcap = rep2(FB);
            int hm16 = 16 * htop(tl1, S);  // H(-1, tlen-1), then down the last column
            const int src_prog_warp = (wg + W - 1) % W;
            const uint32_t edge_x = K.kxa & 0xffffu, edge_x2 = K.kxa2 & 0xffffu;
            const int last_k = qlen + KSW_LAG;
            for (int k0 = 0; k0 < last_k; k0 += 32) {
                if (A.deadline) {
                    // cooperative stop, polled every 32 rows (ksw2_progress.c:30-38 polls
                    // every 256 anti-diagonals); any warp of the group stops the pair
                    int st = 0;
                    if (lane == 0) st = (*stop_flag || aw_deadline_passed(A.deadline)) ? 1 : 0;
                    st = __shfl_sync(FULLMASK, st, 0);
                    if (st) {
                        if (lane == 0) *stop_flag = 1;
                        stopped = true;
                        break;
                    }
                }
                // lane 0's left values for rows k0 .. k0+31, one row per lane, with the
                // row's query code in the top half of the second word
                const int row = k0 + lane;
                uint32_t bx = 0, by = 0;
                if (k0 < qlen) {
                    const uint32_t qc = row < qlen ? (qs[row] & 7u) : 0u;
                    if (s == 0) {
                        bx = edge_x | ((uint32_t)(16 * edge_diff(row, S) + FB) << 16);
                        by = edge_x2 | (qc << 16);
                    } else {
                        const int need = min(k0 + 32, qlen);
                        if (lane == 0) {
                            int spins = 0;
                            cuda::atomic_ref<int, cuda::thread_scope_block> pr(prog[src_prog_warp]);
                            const int target = (s - 1) * C.pstride + need;
                            while (pr.load(cuda::memory_order_acquire) < target) {
                                if (*stop_flag) break;  // the producer stopped at the deadline
                                if (++spins > (1 << 26)) {
                                    atomicExch(A.error, 1);
                                    break;
                                }
                                __nanosleep(32);
                            }
                        }
                        __syncwarp();
                        if (A.deadline) {
                            int st = lane == 0 ? *stop_flag : 0;
                            if (__shfl_sync(FULLMASK, st, 0)) {
                                stopped = true;
                                break;
                            }
                        }
                        if (row < qlen) {
                            const uint2 e = __ldcg(C.bnd + (int64_t)(s - 1) * C.bstride + row);
                            bx = e.x, by = (e.y & 0xffffu) | (qc << 16);
                        }
                    }
                }
                const int k1 = min(k0 + 32, last_k);
                if (last) sweep_range<CIGAR, RIGHT, true>(w, C, k0, k1, bx, by, K, hm16, mte16, mte_q);
                else sweep_range<CIGAR, RIGHT, false>(w, C, k0, k1, bx, by, K, hm16, mte16, mte_q);
            }
            __syncwarp();
            if (stopped) break;
            // last row: H(qlen-1, col) = H(qlen-1, col0 - 1) + the prefix sum of the last
            // row's u (the column state after the sweep) along the strip
            int lsum = 0;
#pragma unroll
            for (int c = 0; c < 8; ++c) lsum += fld(w.U[c], 0) + fld(w.U[c], 1) - 2 * FB;
            int incl = lsum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULLMASK, incl, o);
                if (lane >= o) incl += t;
            }
            int base16 = 0;
            if (s == 0) {
                base16 = 16 * htop(qlen - 1, S);
            } else {
                if (lane == 0) {
                    int spins = 0;
                    cuda::atomic_ref<int, cuda::thread_scope_block> pr(prog[src_prog_warp]);
                    const int target = (s - 1) * C.pstride + qlen + 1;
                    while (pr.load(cuda::memory_order_acquire) < target) {
                        if (*stop_flag) break;
                        if (++spins > (1 << 26)) {
                            atomicExch(A.error, 1);
                            break;
                        }
                        __nanosleep(32);
                    }
                    base16 = (int)__ldcg(C.bnd + (int64_t)(s - 1) * C.bstride + qlen).x;
                }
                base16 = __shfl_sync(FULLMASK, base16, 0);
                if (A.deadline) {
                    int st = lane == 0 ? *stop_flag : 0;
                    if (__shfl_sync(FULLMASK, st, 0)) {
                        stopped = true;
                        break;
                    }
                }
            }
            int h = base16 + incl - lsum;
#pragma unroll
            for (int f = 0; f < 2; ++f) {
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    h += fld(w.U[c], f) - FB;
                    const int col = col0 + 8 * f + c;
                    if (col < tlen) {
                        if (h >= mqe16) mqe16 = h, mqe_t = col;
                        if (col == tl1) score16 = h;
                    }
                }
            }
            if (C.bnd_writer) {
                C.bnd[(int64_t)s * C.bstride + qlen] = make_uint2((uint32_t)h, 0u);
                __threadfence();
                cuda::atomic_ref<int, cuda::thread_scope_block> pw(prog[wg]);
                pw.store(s * C.pstride + qlen + 1, cuda::memory_order_release);
            }
        }
        int mqe = mqe_t >= 0 ? mqe16 >> 4 : AW_NEG_INF;
        int mte = mte_q >= 0 ? mte16 >> 4 : AW_NEG_INF;
        int score = score16 != INT_MIN ? score16 >> 4 : AW_NEG_INF;
        // reduce end tracking over lanes, then over the warps of the group
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int ov = __shfl_xor_sync(FULLMASK, mqe, o), op = __shfl_xor_sync(FULLMASK, mqe_t, o);
            best_merge(mqe, mqe_t, ov, op);
            const int tv = __shfl_xor_sync(FULLMASK, mte, o), tp = __shfl_xor_sync(FULLMASK, mte_q, o);
            best_merge(mte, mte_q, tv, tp);
            score = max(score, __shfl_xor_sync(FULLMASK, score, o));
        }
        if (lane == 0) {
            s_red[warp][0] = mqe, s_red[warp][1] = mqe_t, s_red[warp][2] = mte, s_red[warp][3] = mte_q;
            s_red[warp][4] = score;
        }
        group_sync(g, W * 32);
        if (wg == 0 && lane == 0) {
            for (int w2 = 1; w2 < W; ++w2) {
                const int *rr = s_red[g * W + w2];
                best_merge(mqe, mqe_t, rr[0], rr[1]);
                best_merge(mte, mte_q, rr[2], rr[3]);
                score = max(score, rr[4]);
            }
            KswOut o;
            const int stop = *stop_flag;
            o.score = stop ? AW_NEG_INF : score, o.max = 0, o.max_q = -1, o.max_t = -1;
            o.mqe = mqe, o.mqe_t = mqe_t, o.mte = mte, o.mte_q = mte_q;
            o.n_cigar = 0, o.zdropped = 0, o.reach_end = 0, o.stopped = stop;
            A.out[idx] = o;
        }
    }
}

// ---- traceback -------------------------------------------------------------

// CIGAR under construction, replicated in every lane of the walking warp: the open
// run stays in registers and lane 0 writes a run when the next op differs (the
// merge rule of ksw_push_cigar, minimap2/ksw2.h:144-154).
struct WarpCigar {
    uint32_t *buf;
    int n;
    uint32_t op;
    int len;
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

constexpr int BT_WARPS = 4;

// ksw_backtrack of minimap2/ksw2.h:160-192 over the strip layout; in full mode
// every visited cell is a stored cell, so the off/off_end forcing never fires.
// One warp per pair walks in lockstep and fetches traceback tiles cooperatively.
__global__ void __launch_bounds__(32 * BT_WARPS)
    ksw_backtrack_full_kernel(const KswPair *pairs, const int32_t *order, int n, const uint8_t *tb_arena,
                              KswOut *out, uint32_t *cig, int flag) {
    using Cache = TileCache<8>;
    __shared__ Cache::Word tiles[BT_WARPS][2 * Cache::NW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pi = blockIdx.x * BT_WARPS + warp;
    if (pi >= n) return;
    const int idx = order[pi];
    const KswPair P = pairs[idx];
    KswOut o = out[idx];
    const int qlen = P.qlen, tlen = P.tlen;
    int i0 = tlen - 1, j0 = qlen - 1;
    if (o.zdropped || o.stopped) return;
    if (flag & AW_EZ_SEMIGLOBAL_END) {
        if (o.mqe > o.mte) o.score = o.mqe, i0 = o.mqe_t, j0 = qlen - 1;
        else o.score = o.mte, i0 = tlen - 1, j0 = o.mte_q;
    }
    const uint8_t *tb = tb_arena + P.tb_off;
    const int64_t stride_k = qlen + KSW_LAG;
    Cache cache;
    cache.init(tiles[warp]);
    auto load = [&](int gg, int jj) -> uint2 {
        if (gg < 0 || jj < 0 || jj >= qlen || (gg << 3) >= tlen) return make_uint2(0, 0);
        const int s = gg / KSW_GROUPS, L = gg % KSW_GROUPS;
        return __ldcs(reinterpret_cast<const uint2 *>(
            tb + (((int64_t)s * stride_k + jj + L) * KSW_GROUPS + L) * KSW_COLS));
    };
    WarpCigar w{cig + P.cig_off, 0, 0, 0};
    int i = i0, j = j0, state = 0;
    while (i >= 0 && j >= 0) {
        const uint32_t cellv = cache.byte(i >> 3, j, i & 7, load);
        if (state == 0) state = cellv & 7;
        else if (!(cellv >> (state + 2) & 1)) state = 0;
        if (state == 0) state = cellv & 7;
        if (state == 0) w.push(0, 1), --i, --j;
        else if (state == 1 || state == 3) w.push(2, 1), --i;
        else w.push(1, 1), --j;
    }
    if (i >= 0) w.push(2, i + 1);
    if (j >= 0) w.push(1, j + 1);
    o.n_cigar = w.finish(!(flag & AW_EZ_REV_CIGAR));
    if (lane == 0) out[idx] = o;
}

// Copy each pair's CIGAR from its slot to a packed buffer (one warp per pair).
__global__ void ksw_pack_cigar_kernel(const KswPair *pairs, int n, const KswOut *out,
                                      const uint32_t *cig, const int64_t *packed_off,
                                      uint32_t *packed) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (wid >= n) return;
    const int nc = out[wid].n_cigar;
    const uint32_t *src = cig + pairs[wid].cig_off;
    uint32_t *dst = packed + packed_off[wid];
    for (int i = lane; i < nc; i += 32) dst[i] = src[i];
}

// Dynamic shared memory of a CTA: the score profiles of its warps.
inline int prof_bytes(int warps) { return warps * PROF_WARP; }

template <bool CIGAR, bool RIGHT, int W>
cudaError_t launch_t(const KswFullArgs &a, int groups, int ctas, cudaStream_t st) {
    const int smem = prof_bytes(groups * W);
    // the dynamic shared memory limit is an attribute of the kernel on a device: set once
    static std::atomic<uint32_t> set_on(0);
    int dev = 0;
    cudaGetDevice(&dev);
    const uint32_t bit = 1u << (dev & 31);
    if (!(set_on.load() & bit)) {
        cudaError_t e = cudaFuncSetAttribute(ksw_full_kernel<CIGAR, RIGHT, W>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, prof_bytes(8));
        if (e != cudaSuccess) return e;
        set_on.fetch_or(bit);
    }
    ksw_full_kernel<CIGAR, RIGHT, W><<<ctas, groups * W * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool CIGAR, bool RIGHT>
cudaError_t launch_w(const KswFullArgs &a, int W, int groups, int ctas, cudaStream_t st) {
    switch (W) {
    case 1: return launch_t<CIGAR, RIGHT, 1>(a, groups, ctas, st);
    case 2: return launch_t<CIGAR, RIGHT, 2>(a, groups, ctas, st);
    case 4: return launch_t<CIGAR, RIGHT, 4>(a, groups, ctas, st);
    case 8: return launch_t<CIGAR, RIGHT, 8>(a, groups, ctas, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int ksw_full_occupancy(int flag, int warps_per_pair, int groups_per_cta) {
    // CTAs per SM depend only on the instantiation and the CTA shape: cached per device
    static std::atomic<int> cache[16][3][4][4];
    int dev = 0;
    cudaGetDevice(&dev);
    const int mode = (flag & AW_EZ_SCORE_ONLY) ? 0 : (flag & AW_EZ_RIGHT) ? 2 : 1;
    const int wi = warps_per_pair == 1 ? 0 : warps_per_pair == 2 ? 1 : warps_per_pair == 4 ? 2 : 3;
    const int gi = groups_per_cta == 1 ? 0 : groups_per_cta == 2 ? 1 : groups_per_cta == 4 ? 2 : 3;
    std::atomic<int> *slot = dev >= 0 && dev < 16 ? &cache[dev][mode][wi][gi] : nullptr;
    if (slot && slot->load() > 0) return slot->load();
    int nb = 0;
    const int threads = warps_per_pair * groups_per_cta * 32;
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY), right = !!(flag & AW_EZ_RIGHT);
    cudaError_t e = cudaErrorInvalidValue;
#define AW_OCC(CG, RT, WW)                                                                                   \
    cudaFuncSetAttribute(ksw_full_kernel<CG, RT, WW>, cudaFuncAttributeMaxDynamicSharedMemorySize, prof_bytes(8)); \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ksw_full_kernel<CG, RT, WW>, threads,                   \
                                                      prof_bytes(warps_per_pair * groups_per_cta))
#define AW_OCC_W(CG, RT)                                                 \
    switch (warps_per_pair) {                                            \
    case 1: AW_OCC(CG, RT, 1); break;                                    \
    case 2: AW_OCC(CG, RT, 2); break;                                    \
    case 4: AW_OCC(CG, RT, 4); break;                                    \
    case 8: AW_OCC(CG, RT, 8); break;                                    \
    }
    if (cigar && right) { AW_OCC_W(true, true) }
    else if (cigar) { AW_OCC_W(true, false) }
    else { AW_OCC_W(false, false) }
#undef AW_OCC_W
#undef AW_OCC
    if (e != cudaSuccess) return 0;
    if (slot) slot->store(nb);
    return nb;
}

cudaError_t launch_ksw_full(const KswFullArgs &a, int flag, int warps_per_pair, int groups_per_cta,
                            int ctas, cudaStream_t st) {
    if (warps_per_pair * groups_per_cta > 8 || warps_per_pair * groups_per_cta < 1)
        return cudaErrorInvalidValue;
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY), right = !!(flag & AW_EZ_RIGHT);
    if (cigar && right) return launch_w<true, true>(a, warps_per_pair, groups_per_cta, ctas, st);
    if (cigar) return launch_w<true, false>(a, warps_per_pair, groups_per_cta, ctas, st);
    return launch_w<false, false>(a, warps_per_pair, groups_per_cta, ctas, st);
}

cudaError_t launch_ksw_backtrack_full(const KswPair *pairs, const int32_t *order, int n,
                                      const uint8_t *tb, KswOut *out, uint32_t *cig, int flag,
                                      cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    ksw_backtrack_full_kernel<<<(n + BT_WARPS - 1) / BT_WARPS, 32 * BT_WARPS, 0, st>>>(pairs, order, n, tb, out,
                                                                                       cig, flag);
    return cudaGetLastError();
}

__global__ void set_deadline_kernel(unsigned long long *d, unsigned long long remaining_ns) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *d = remaining_ns == ~0ull ? ~0ull : t + remaining_ns;
}

cudaError_t launch_set_deadline(unsigned long long *deadline, unsigned long long remaining_ns, cudaStream_t st) {
    set_deadline_kernel<<<1, 1, 0, st>>>(deadline, remaining_ns);
    return cudaGetLastError();
}

cudaError_t launch_ksw_pack_cigar(const KswPair *pairs, int n, const KswOut *out,
                                  const uint32_t *cig, const int64_t *packed_off, uint32_t *packed,
                                  cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const int blocks = (int)(((int64_t)n * 32 + threads - 1) / threads);
    ksw_pack_cigar_kernel<<<blocks, threads, 0, st>>>(pairs, n, out, cig, packed_off, packed);
    return cudaGetLastError();
}

}  // namespace aw
