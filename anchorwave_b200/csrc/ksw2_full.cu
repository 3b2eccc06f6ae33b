// KSW2 extd2, full-matrix form (w < 0 or w >= max(qlen, tlen)), on sm_100a.
//
// Same recurrence as minimap2/ksw2_extd2_sse.c:43-71 + :237-330 (difference-
// encoded u, v, x, y, x2, y2 cells; state byte d with the 3-bit argmax and the
// four continuation bits), computed cell by cell in 32-bit registers.  In full
// mode every cell the recurrence reads is a real matrix cell or a matrix edge,
// so the SIMD padding lanes of the reference never influence the result and
// are not computed here.  The host only routes parameter sets to this kernel
// whose int8 intermediates provably cannot wrap (ksw2_api.cu: full_path_ok).
//
// Work decomposition (one pair per group of W warps):
//   * target columns are cut into strips of 256 (32 lanes x 8 columns);
//   * a warp sweeps the query rows of its strip with a one-row skew per lane:
//     at step k lane L owns row j = k - L, so the (x, v, x2) values of a lane's
//     last column reach the next lane by one __shfl_up per step, together with
//     the query code of that row;
//   * strip s+1 takes its left edge (column 256(s+1)-1 of strip s) from a
//     global boundary buffer that strip s fills row by row; with W > 1 the W
//     warps of a group run consecutive strips concurrently, the consumer warp
//     polling the producer's published row count in shared memory (bounded);
//   * traceback bytes go to HBM as one coalesced 256-byte store per warp-step,
//     with evict-first policy (they are read back only along one path).
// Pairs are pulled from a device work queue (atomicAdd on a head counter) in
// the host-provided order (largest first), so one persistent launch serves a
// whole batch of uneven pairs.
#include "aw_internal.h"
#include "tb_walk.cuh"
#include <cuda/atomic>

namespace aw {

namespace {

constexpr int MAX_GROUP_WARPS = 32;

__device__ __forceinline__ int prmt_sx(uint32_t lo, uint32_t hi, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return (int)r;
}

__device__ __forceinline__ int sx8(uint32_t w) { return (int)(int8_t)(uint8_t)w; }

__device__ __forceinline__ uint32_t pack3(int a, int b, int c, uint32_t top) {
    return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) |
           (top << 24);
}

// Difference along a matrix edge for edge cell index r (ksw2_extd2_sse.c:167,171).
__device__ __forceinline__ int edge_diff(int r, const KswScore &S) {
    return r == 0 ? -S.qe : r < S.long_thres ? -S.e : r == S.long_thres ? S.long_diff : -S.e2;
}

// H(t, -1): sum of edge_diff(0..t), the score of a leading gap of length t+1,
// offset as the reference's H[0] = v[0] - qe with qe taken before the swap.
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

#ifndef AW_CELL_DPX
#define AW_CELL_DPX 2
#endif
#ifndef AW_ARGMAX_DPX
#define AW_ARGMAX_DPX 1
#endif

template <bool CIGAR, bool RIGHT>
__device__ __forceinline__ void cell(int s, int &xs, int &vs, int &x2s, int &ut, int &yt, int &y2t,
                                     int &d, const KswScore &S) {
    int a = xs + vs, b = yt + ut, a2 = x2s + vs, b2 = y2t + ut;
    int z = s;
#if AW_CELL_DPX && AW_ARGMAX_DPX
    // Arg-max chain with the reference's tie rules, one DPX max+predicate per step:
    // left-aligned takes a candidate only if strictly greater (ksw2_extd2_sse.c:244-251),
    // right-aligned also on equality (:291-298).
    bool p;
    if (!CIGAR) {
        z = __vimax3_s32(z, a, b);
        z = __vimax3_s32(z, a2, b2);
    } else if (!RIGHT) {
        z = __vibmax_s32(z, a, &p);  // p = z >= a
        d = p ? 0 : 1;
        z = __vibmax_s32(z, b, &p);
        d = p ? d : 2;
        z = __vibmax_s32(z, a2, &p);
        d = p ? d : 3;
        z = __vibmax_s32(z, b2, &p);
        d = p ? d : 4;
    } else {
        z = __vibmax_s32(a, z, &p);  // p = a >= z
        d = p ? 1 : 0;
        z = __vibmax_s32(b, z, &p);
        d = p ? 2 : d;
        z = __vibmax_s32(a2, z, &p);
        d = p ? 3 : d;
        z = __vibmax_s32(b2, z, &p);
        d = p ? 4 : d;
    }
#else
    if (!CIGAR) {
        z = max(max(max(z, a), max(b, a2)), b2);
    } else if (!RIGHT) {
        d = a > z ? 1 : 0;
        z = max(z, a);
        d = b > z ? 2 : d;
        z = max(z, b);
        d = a2 > z ? 3 : d;
        z = max(z, a2);
        d = b2 > z ? 4 : d;
        z = max(z, b2);
    } else {
        d = z > a ? 0 : 1;
        z = max(z, a);
        d = z > b ? d : 2;
        z = max(z, b);
        d = z > a2 ? d : 3;
        z = max(z, a2);
        d = z > b2 ? d : 4;
        z = max(z, b2);
    }
#endif
    z = min(z, S.mch);
    const int un = z - vs, vn = z - ut;
#if AW_CELL_DPX >= 2
    if (!(CIGAR && RIGHT)) {
        // x' = max(a - z + q, 0) - (q + e) = max(a + (-e - z), -(q + e)): one add+max each
        const int nez = -S.e - z, nez2 = -S.e2 - z;
        xs = __viaddmax_s32(a, nez, -S.qe);
        yt = __viaddmax_s32(b, nez, -S.qe);
        x2s = __viaddmax_s32(a2, nez2, -S.qe2);
        y2t = __viaddmax_s32(b2, nez2, -S.qe2);
        if (CIGAR) {
            // continuation bit (a - z + q > 0) == (x' + q + e > 0) == min(x' + q + e, 1)
            d += 0x08 * __viaddmin_s32(xs, S.qe, 1);
            d += 0x10 * __viaddmin_s32(yt, S.qe, 1);
            d += 0x20 * __viaddmin_s32(x2s, S.qe2, 1);
            d += 0x40 * __viaddmin_s32(y2t, S.qe2, 1);
        }
        ut = un;
        vs = vn;
        return;
    }
#endif
    a = a - z + S.q;
    b = b - z + S.q;
    a2 = a2 - z + S.q2;
    b2 = b2 - z + S.q2;
    xs = max(a, 0) - S.qe;
    yt = max(b, 0) - S.qe;
    x2s = max(a2, 0) - S.qe2;
    y2t = max(b2, 0) - S.qe2;
    if (CIGAR) {
        if (!RIGHT)
            d |= (a > 0 ? 0x08 : 0) | (b > 0 ? 0x10 : 0) | (a2 > 0 ? 0x20 : 0) | (b2 > 0 ? 0x40 : 0);
        else
            d |= (a >= 0 ? 0x08 : 0) | (b >= 0 ? 0x10 : 0) | (a2 >= 0 ? 0x20 : 0) | (b2 >= 0 ? 0x40 : 0);
    }
    ut = un;
    vs = vn;
}

// Lexicographic (value, position) maximum: later positions win ties, the
// ">=" end-tracking rule of ksw2_extd2_sse.c:369-372.
__device__ __forceinline__ void best_merge(int &v, int &p, int ov, int op) {
    if (ov > v || (ov == v && op > p)) v = ov, p = op;
}

template <bool CIGAR, bool RIGHT, int W>
__global__ void __launch_bounds__(256) ksw_full_kernel(KswFullArgs A) {
    constexpr int C = KSW_COLS;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = warp / W;
    const int wg = warp % W;
    const KswScore &S = A.sc;
    __shared__ int s_pair[MAX_GROUP_WARPS];
    __shared__ int s_prog[MAX_GROUP_WARPS];           // rows published, per warp (monotone per pair)
    __shared__ int s_red[MAX_GROUP_WARPS][5];
    __shared__ int s_stop[MAX_GROUP_WARPS];           // the group's pair passed the deadline
    int *prog = s_prog + g * W;
    volatile int *stop_flag = s_stop + g;

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
        uint32_t *bnd = A.bnd + P.bnd_off;
        uint8_t *tb = CIGAR ? A.tb + P.tb_off : nullptr;
        const int nstrip = (tlen + KSW_STRIP - 1) / KSW_STRIP;
        const int stride_k = qlen + 31;
        int mqe = AW_NEG_INF, mqe_t = -1, mte = AW_NEG_INF, mte_q = -1, score = AW_NEG_INF;
        bool stopped = false;

        for (int s = wg; s < nstrip && !stopped; s += W) {
            const int col0 = s * KSW_STRIP + lane * C;
            int ut[C], yt[C], y2t[C], H[C];
            uint32_t rlo[C], rhi[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int col = col0 + c;
                const int tc = col < tlen ? (ts[col] & 7) : 0;
                rlo[c] = S.tab_lo[tc];
                rhi[c] = S.tab_hi[tc];
                ut[c] = edge_diff(col, S);
                yt[c] = -S.qe;
                y2t[c] = -S.qe2;
                H[c] = htop(col, S);
            }
            // rows of the previous strip must be published before we read them
            const int src_prog_warp = (wg + W - 1) % W;
            uint32_t carry = 0, qchunk = 0, bchunk = 0;
            const int last_k = qlen + 31;
            for (int k = 0; k < last_k; ++k) {
                if ((k & 31) == 0 && A.deadline) {
                    // cooperative stop, polled every 32 rows (ksw2_progress.c:30-38 polls
                    // every 256 anti-diagonals); any warp of the group stops the pair
                    int st = 0;
                    if (lane == 0) st = (*stop_flag || aw_deadline_passed(A.deadline)) ? 1 : 0;
                    st = __shfl_sync(0xffffffffu, st, 0);
                    if (st) {
                        if (lane == 0) *stop_flag = 1;
                        stopped = true;
                        break;
                    }
                }
                if ((k & 31) == 0 && k < qlen) {
                    const int J = k;
                    qchunk = (J + lane < qlen) ? qs[J + lane] : 0u;
                    if (s > 0) {
                        const int need = min(J + 32, qlen);
                        int spins = 0;
                        cuda::atomic_ref<int, cuda::thread_scope_block> pr(prog[src_prog_warp]);
                        // the producer publishes (strip, rows) as strip*(qlen+1)+rows
                        const int target = (s - 1) * (qlen + 1) + need;
                        while (pr.load(cuda::memory_order_acquire) < target) {
                            if (*stop_flag) break;  // the producer stopped at the deadline
                            if (++spins > (1 << 26)) {
                                atomicExch(A.error, 1);
                                break;
                            }
                            __nanosleep(32);
                        }
                        if (A.deadline) {
                            int st = lane == 0 ? *stop_flag : 0;
                            st = __shfl_sync(0xffffffffu, st, 0);
                            if (st) {
                                stopped = true;
                                break;
                            }
                        }
                        bchunk = (J + lane < qlen) ? __ldcg(bnd + (int64_t)(s - 1) * qlen + J + lane) : 0u;
                    }
                }
                const uint32_t qv = __shfl_sync(0xffffffffu, qchunk, k & 31);
                const uint32_t bv = __shfl_sync(0xffffffffu, bchunk, k & 31);
                const uint32_t in = __shfl_up_sync(0xffffffffu, carry, 1);
                const int j = k - lane;
                int xs, vs, x2s;
                uint32_t qc;
                if (lane == 0) {
                    qc = qv & 7u;
                    if (s == 0) {
                        xs = -S.qe, x2s = -S.qe2, vs = edge_diff(j, S);
                    } else {
                        xs = sx8(bv), vs = sx8(bv >> 8), x2s = sx8(bv >> 16);
                    }
                } else {
                    qc = in >> 24;
                    xs = sx8(in), vs = sx8(in >> 8), x2s = sx8(in >> 16);
                }
                if (j >= 0 && j < qlen) {
                    const uint32_t sel = qc * 0x1111u + 0x8880u;
                    uint32_t dlo = 0, dhi = 0;
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        int d = 0;
                        const int sc = prmt_sx(rlo[c], rhi[c], sel);
                        cell<CIGAR, RIGHT>(sc, xs, vs, x2s, ut[c], yt[c], y2t[c], d, S);
                        H[c] += vs;
                        if (CIGAR) {
                            if (c < 4) dlo |= (uint32_t)d << (8 * c);
                            else dhi |= (uint32_t)d << (8 * (c - 4));
                        }
                    }
                    carry = pack3(xs, vs, x2s, qc);
                    if (CIGAR) {
                        uint2 *dst = reinterpret_cast<uint2 *>(tb + (((int64_t)s * stride_k + k) * 32 + lane) * C);
                        __stcs(dst, make_uint2(dlo, dhi));
                    }
                    if (j == qlen - 1) {
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const int col = col0 + c;
                            if (col < tlen && H[c] >= mqe) mqe = H[c], mqe_t = col;
                        }
                    }
                    const int cl = tlen - 1 - col0;
                    if (cl >= 0 && cl < C) {
                        int hv = H[0];
#pragma unroll
                        for (int c = 1; c < C; ++c)
                            if (c == cl) hv = H[c];
                        if (hv >= mte) mte = hv, mte_q = j;
                        if (j == qlen - 1) score = hv;
                    }
                    if (lane == 31 && s + 1 < nstrip) bnd[(int64_t)s * qlen + j] = pack3(xs, vs, x2s, 0);
                }
                if (lane == 31 && s + 1 < nstrip) {
                    const int jj = k - 31;
                    if (jj >= 0 && ((jj & 31) == 31 || jj == qlen - 1)) {
                        // the consumer reads these rows from L2 (ld.cg), so they must be
                        // visible at device scope before the row count is published
                        __threadfence();
                        cuda::atomic_ref<int, cuda::thread_scope_block> pw(prog[wg]);
                        pw.store(s * (qlen + 1) + jj + 1, cuda::memory_order_release);
                    }
                }
            }
            __syncwarp();
        }
        // reduce end tracking over lanes, then over the warps of the group
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int ov = __shfl_xor_sync(0xffffffffu, mqe, o), op = __shfl_xor_sync(0xffffffffu, mqe_t, o);
            best_merge(mqe, mqe_t, ov, op);
            const int tv = __shfl_xor_sync(0xffffffffu, mte, o), tp = __shfl_xor_sync(0xffffffffu, mte_q, o);
            best_merge(mte, mte_q, tv, tp);
            score = max(score, __shfl_xor_sync(0xffffffffu, score, o));
        }
        if (lane == 0) {
            s_red[warp][0] = mqe, s_red[warp][1] = mqe_t, s_red[warp][2] = mte, s_red[warp][3] = mte_q;
            s_red[warp][4] = score;
        }
        group_sync(g, W * 32);
        if (wg == 0 && lane == 0) {
            for (int w = 1; w < W; ++w) {
                const int *rr = s_red[g * W + w];
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
    const int64_t stride_k = qlen + 31;
    Cache cache;
    cache.init(tiles[warp]);
    auto load = [&](int gg, int jj) -> uint2 {
        if (gg < 0 || jj < 0 || jj >= qlen || (gg << 3) >= tlen) return make_uint2(0, 0);
        const int s = gg >> 5, L = gg & 31;
        return __ldcs(reinterpret_cast<const uint2 *>(tb + (((int64_t)s * stride_k + jj + L) * 32 + L) * KSW_COLS));
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

template <bool CIGAR, bool RIGHT, int W>
cudaError_t launch_t(const KswFullArgs &a, int groups, int ctas, cudaStream_t st) {
    ksw_full_kernel<CIGAR, RIGHT, W><<<ctas, groups * W * 32, 0, st>>>(a);
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
    int nb = 0;
    const int threads = warps_per_pair * groups_per_cta * 32;
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY), right = !!(flag & AW_EZ_RIGHT);
    cudaError_t e = cudaErrorInvalidValue;
#define AW_OCC(CG, RT, WW) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ksw_full_kernel<CG, RT, WW>, threads, 0)
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
    return e == cudaSuccess ? nb : 0;
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
