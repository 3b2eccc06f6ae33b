// The sequence pass of AnchorWave's alignment selector on the device:
// summarizeSequencePair (src/myImportandFunction/AlignmentAlgorithmSelector.cpp:730-757)
// over SequenceProfileAccumulator (:591-728) for a batch of interval pairs.
//
// Per sequence the reference walks the bases once, keeping a rolling 2-bit k-mer for
// k = 9, 15, 21 (reset by any base other than A/C/G/T in either case), and collects
//   * the k-mers whose mixHash (:561-568) is divisible by the scale's sampling modulo,
//     in position order, at most 4 entries per hash value (:640-660);
//   * the fraction of other bases, the fraction of bases at run length >= 4 of one base,
//     and the entropy of each 64-base block (Shannon entropy of its A/C/G/T counts / 2 x
//     its A/C/G/T bases, summed and divided by the length, :672-700);
//   * an FNV-1a fingerprint of the bytes (byte-serial: computed by host threads while the
//     device works) and the identity of the two sequences.
//
// Device layout: the 2n sequences back to back; tiles of 1024 positions, one CTA each,
// with the 20 preceding bases as halo in shared memory. Every position is independent
// given its 21-base window, so the rolling state of the reference becomes a per-thread
// window over shared memory.
//   1. count pass: composition counters and entropy per sequence (atomics), sampled
//      k-mers per tile and scale;
//   2. exclusive scans of the tile counts -> each (sequence, scale) owns a contiguous
//      range of candidates in position order;
//   3. emit pass (per chunk of sequences, sized so that candidates and tables fit a
//      budget): the candidates at their ranks;
//   4. cap pass, one warp per (sequence, scale): candidates in order, 32 at a time; an
//      entry is kept while fewer than 4 earlier candidates have its hash (equal hashes in
//      the same 32 by __match_any_sync, earlier ones by an open-addressing table in global
//      memory); kept entries are compacted in place;
//   5. gather of the kept entries into one output array.
#include "aw_internal.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace aw {
namespace {

constexpr int SUM_TILE = 1024;
constexpr int SUM_HALO = 20;  // k_max - 1
constexpr int SUM_THREADS = 256;
constexpr int SUM_PER_THREAD = SUM_TILE / SUM_THREADS;  // 4 consecutive positions
// entropy blocks of 64 bases: 16 threads each
constexpr uint32_t SUM_MAX_OCC = 4;
constexpr uint64_t SUM_TARGET[3] = {1024, 4096, 1024};

// Divisibility by a sampling modulo d = d0 * 2^s (d0 odd) without a division
// (Granlund & Montgomery, "Division by invariant integers using multiplication", 1994;
// Warren, Hacker's Delight, 2nd ed., 10-17): d | h exactly when
// rotr(h * d0^-1 mod 2^64, s) <= floor((2^64 - 1) / d).
struct DivTest {
    uint64_t inv, limit;
    uint32_t shift, pad;
};

struct SeqDev {
    int64_t off, len;
    DivTest div[3];
    int32_t first_tile, ntiles;
};

// k of scale sc: 9, 15, 21
__host__ __device__ __forceinline__ uint64_t kmer_len(int sc) { return (uint64_t)(9 + 6 * sc); }

__device__ __forceinline__ uint64_t mix_hash(uint64_t v) {
    v ^= v >> 30;
    v *= 0xbf58476d1ce4e5b9ULL;
    v ^= v >> 27;
    v *= 0x94d049bb133111ebULL;
    v ^= v >> 31;
    return v;
}

__device__ __forceinline__ bool divisible(uint64_t h, const DivTest &d) {
    uint64_t x = h * d.inv;
    if (d.shift) x = (x >> d.shift) | (x << (64 - d.shift));
    return x <= d.limit;
}

__device__ __forceinline__ int8_t base_code(uint8_t b) {
    const uint8_t u = (b >= 'a' && b <= 'z') ? (uint8_t)(b - 32) : b;
    return u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : -1;
}

// Block-wide exclusive scan of one value per thread (256 threads); returns the prefix,
// *total the sum.
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t *warp_sums, uint32_t *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < SUM_THREADS / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        if (lane < SUM_THREADS / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (w ? warp_sums[w - 1] : 0u) + x - v;
    *total = warp_sums[SUM_THREADS / 32 - 1];
    __syncthreads();
    return before;
}

// One tile of one sequence. COUNT: composition, entropy and sampled-k-mer counts.
// Otherwise: the sampled k-mers of the tile, written at their ranks.
template <bool COUNT>
__global__ void __launch_bounds__(SUM_THREADS) summary_tile_kernel(
    const uint8_t *bases, const SeqDev *seqs, const int32_t *tile_seq, int32_t tile0, int64_t ntiles_all,
    unsigned long long *amb, unsigned long long *tail, double *entropy /* per tile */, uint32_t *tile_cnt,
    const int64_t *tile_off, const int64_t *chunk_first, const int64_t *chunk_base, uint64_t *cand_hash,
    uint32_t *cand_pos) {
    __shared__ int8_t code[SUM_TILE + SUM_HALO];
    __shared__ uint32_t warp_sums[SUM_THREADS / 32];
    const int64_t t = (int64_t)tile0 + blockIdx.x;
    const int j = tile_seq[t];
    const SeqDev S = seqs[j];
    const int64_t p0 = (int64_t)(t - S.first_tile) * SUM_TILE;
    for (int i = threadIdx.x; i < SUM_TILE + SUM_HALO; i += SUM_THREADS) {
        const int64_t p = p0 - SUM_HALO + i;
        code[i] = (p < 0 || p >= S.len) ? (int8_t)-2 : base_code(bases[S.off + p]);
    }
    __syncthreads();
    const int tid = threadIdx.x;
    // 21-base window ending at each of this thread's positions: valid run and k-mer
    uint32_t run = 0;
    uint64_t val = 0;
    uint32_t nsamp[3] = {0, 0, 0};
    uint64_t sh[SUM_PER_THREAD][3];
    bool sf[SUM_PER_THREAD][3];
    uint32_t cnt[5] = {0, 0, 0, 0, 0}, nb = 0, ntail = 0;
#pragma unroll
    for (int m = 0; m < SUM_HALO + SUM_PER_THREAD; ++m) {
        const int8_t c = code[SUM_PER_THREAD * tid + m];
        if (c < 0) run = 0, val = 0;
        else run = min(run + 1, 32u), val = ((val << 2) | (uint64_t)c) & ((1ULL << 42) - 1);
        if (m < SUM_HALO) continue;
        const int u = m - SUM_HALO;
        const int64_t p = p0 + SUM_PER_THREAD * tid + u;
#pragma unroll
        for (int sc = 0; sc < 3; ++sc) sf[u][sc] = false, sh[u][sc] = 0;
        if (p >= S.len) continue;
        if (COUNT) {
            ++nb;
#pragma unroll
            for (int b = 0; b < 4; ++b) cnt[b] += c == b;
            if (c < 0) ++cnt[4];
            else {
                // run length >= 4 of one base (the reference's runLength_)
                const int8_t *w = &code[SUM_PER_THREAD * tid + m];
                if (w[-1] == c && w[-2] == c && w[-3] == c) ++ntail;
            }
        }
#pragma unroll
        for (int sc = 0; sc < 3; ++sc) {
            const uint64_t k = kmer_len(sc);
            if (run < k) continue;
            const uint64_t h = mix_hash(val & ((1ULL << (2 * k)) - 1));
            if (divisible(h, S.div[sc])) sf[u][sc] = true, sh[u][sc] = h, ++nsamp[sc];
        }
    }
    if (COUNT) {
        // 16 threads per 64-base block: reduce its counts, one thread adds its entropy
        uint32_t v[6] = {cnt[0], cnt[1], cnt[2], cnt[3], cnt[4], nb};
#pragma unroll
        for (int d = 8; d >= 1; d >>= 1)
#pragma unroll
            for (int i = 0; i < 6; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], d);
        // the tile's 16 blocks summed in order (and the tiles in order per sequence
        // later), so that the result does not depend on scheduling
        __shared__ double ent_blk[SUM_TILE / 64];
        if ((tid & 15) == 0) {
            double ent = 0.0;
            const uint32_t valid = v[0] + v[1] + v[2] + v[3];
            if (v[5] > 0 && valid) {
                for (int b = 0; b < 4; ++b) {
                    if (!v[b]) continue;
                    const double pr = (double)v[b] / (double)valid;
                    ent -= pr * log2(pr);
                }
                ent = ent / 2.0 * (double)valid / (double)v[5];
            }
            ent_blk[tid >> 4] = ent * (double)v[5];
        }
        __syncthreads();
        if (tid == 0) {
            double e = 0.0;
            for (int b = 0; b < SUM_TILE / 64; ++b) e += ent_blk[b];
            entropy[t] = e;
        }
        uint32_t a = cnt[4], tl = ntail;
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, d);
            tl += __shfl_xor_sync(0xffffffffu, tl, d);
        }
        if ((tid & 31) == 0) {
            if (a) atomicAdd(&amb[j], (unsigned long long)a);
            if (tl) atomicAdd(&tail[j], (unsigned long long)tl);
        }
#pragma unroll
        for (int sc = 0; sc < 3; ++sc) {
            uint32_t total;
            block_scan(nsamp[sc], warp_sums, &total);
            if (tid == 0) tile_cnt[sc * ntiles_all + t] = total;
        }
    } else {
#pragma unroll
        for (int sc = 0; sc < 3; ++sc) {
            uint32_t total;
            uint32_t r = block_scan(nsamp[sc], warp_sums, &total);
            const int64_t base = chunk_base[sc] + (tile_off[sc * (ntiles_all + 1) + t] - chunk_first[sc]);
#pragma unroll
            for (int u = 0; u < SUM_PER_THREAD; ++u)
                if (sf[u][sc]) {
                    cand_hash[base + r] = sh[u][sc];
                    cand_pos[base + r] = (uint32_t)(p0 + SUM_PER_THREAD * tid + u + 1 - (int64_t)kmer_len(sc));
                    ++r;
                }
        }
    }
}

// Exclusive scan of each row of a [rows][n] array into [rows][n + 1] (total last).
__global__ void __launch_bounds__(1024) scan_rows_kernel(const uint32_t *in, int64_t *out, int64_t n) {
    __shared__ int64_t part[1024];
    const uint32_t *a = in + (int64_t)blockIdx.x * n;
    int64_t *o = out + (int64_t)blockIdx.x * (n + 1);
    const int64_t per = (n + 1023) / 1024;
    const int64_t b = threadIdx.x * per, e = min(n, b + per);
    int64_t s = 0;
    for (int64_t i = b; i < e; ++i) s += a[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const int64_t add = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    int64_t run = part[threadIdx.x] - s;
    for (int64_t i = b; i < e; ++i) o[i] = run, run += a[i];
    if (threadIdx.x == 1023) o[n] = part[1023];
}

// Candidate range of every (sequence, scale); entropy sum of every sequence (its tiles
// in order).
__global__ void segments_kernel(const SeqDev *seqs, int nseq, const int64_t *tile_off, int64_t ntiles_all,
                                int64_t *seg_start, int64_t *seg_cnt, const double *tile_ent, double *seq_ent) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nseq) return;
    const SeqDev S = seqs[j];
    double e = 0.0;
    for (int32_t k = 0; k < S.ntiles; ++k) e += tile_ent[S.first_tile + k];
    seq_ent[j] = e;
    for (int sc = 0; sc < 3; ++sc) {
        const int64_t *row = tile_off + sc * (ntiles_all + 1);
        seg_start[3 * j + sc] = row[S.first_tile];
        seg_cnt[3 * j + sc] = row[S.first_tile + S.ntiles] - row[S.first_tile];
    }
}

struct SegDev {
    int64_t cand;   // first candidate in the chunk's arrays
    int64_t count;  // candidates
    int64_t table;  // first slot of its table
    int64_t tsize;  // slots (a power of two)
};

// One warp per (sequence, scale): keep the candidates that have fewer than 4 earlier
// candidates of the same hash (kMaximumOccurrencesPerHash, :647-656); compact in place.
__global__ void cap_kernel(const SegDev *segs, int nseg, uint64_t *cand_hash, uint32_t *cand_pos,
                           unsigned long long *tkey, uint32_t *tcnt, uint32_t *kept) {
    const int g = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= nseg) return;
    const SegDev G = segs[g];
    unsigned long long *key = tkey + G.table;
    uint32_t *cnt = tcnt + G.table;
    const uint64_t tmask = (uint64_t)G.tsize - 1;
    const int tbits = 63 - __clzll((long long)G.tsize);
    const uint32_t lt = (1u << lane) - 1u;
    int64_t nk = 0;
    for (int64_t b = 0; b < G.count; b += 32) {
        const int64_t i = b + lane;
        const bool act = i < G.count;
        uint64_t h = 0;
        uint32_t pos = 0;
        if (act) h = cand_hash[G.cand + i], pos = cand_pos[G.cand + i];
        const unsigned amask = __ballot_sync(0xffffffffu, act);
        const unsigned peers = __match_any_sync(0xffffffffu, h) & amask;
        // earlier candidates of this hash: in the table, and in this group of 32
        uint32_t prior = 0;
        int64_t slot = -1;
        if (act) {
            uint64_t s = (h * 0x9E3779B97F4A7C15ULL) >> (64 - tbits);
            if (tbits == 0) s = 0;
            for (uint64_t probe = 0; probe <= tmask; ++probe, s = (s + 1) & tmask) {
                const uint32_t c = cnt[s];
                if (c == 0) break;
                if (key[s] == h) {
                    prior = c, slot = (int64_t)s;
                    break;
                }
            }
        }
        const bool keep = act && prior + (uint32_t)__popc(peers & lt) < SUM_MAX_OCC;
        __syncwarp();
        // the lowest lane of each hash updates or inserts its count
        if (act && (peers & lt) == 0) {
            const uint32_t add = (uint32_t)__popc(peers);
            if (slot >= 0) {
                cnt[slot] = min(prior + add, 255u);
            } else {
                uint64_t s = (h * 0x9E3779B97F4A7C15ULL) >> (64 - tbits);
                if (tbits == 0) s = 0;
                for (uint64_t probe = 0; probe <= tmask; ++probe, s = (s + 1) & tmask)
                    if (atomicCAS(&cnt[s], 0u, min(add, 255u)) == 0u) {
                        key[s] = h;
                        break;
                    }
            }
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) {
            const int64_t o = G.cand + nk + __popc(km & lt);
            cand_hash[o] = h, cand_pos[o] = pos;
        }
        nk += __popc(km);
        __syncwarp();
    }
    if (lane == 0) kept[g] = (uint32_t)nk;
}

// One warp per segment: kept entries to the output arrays.
__global__ void gather_kernel(const SegDev *segs, int nseg, const int64_t *out_off, const uint64_t *cand_hash,
                              const uint32_t *cand_pos, const uint32_t *kept, uint64_t *out_hash,
                              uint32_t *out_pos) {
    const int g = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= nseg) return;
    const int64_t src = segs[g].cand, dst = out_off[g];
    for (int64_t i = lane; i < kept[g]; i += 32) out_hash[dst + i] = cand_hash[src + i], out_pos[dst + i] = cand_pos[src + i];
}

// Page-locked host buffer that only grows (copies to and from it run at full link rate).
struct PinnedBytes {
    uint8_t *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr, cap = 0;
        const size_t want = std::max(n + n / 4, (size_t)1 << 20);
        const cudaError_t e = cudaMallocHost((void **)&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T> T *as() const { return (T *)p; }
    ~PinnedBytes() {
        if (p) cudaFreeHost(p);
    }
};

struct SummaryBuffers {
    PinnedBytes staging;
    DevBuf bases, seqs, tile_seq, amb, tail, ent, tile_ent, tile_cnt, tile_off, seg_start, seg_cnt;
    DevBuf chunk_first, chunk_base, cand_hash, cand_pos, segs, tkey, tcnt, kept, out_off, out_hash, out_pos;
    PinnedBytes sk_hash, sk_pos;  // the last call's sketch entries
    int64_t sk_n = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~SummaryBuffers() {
        for (DevBuf *b : {&bases, &seqs, &tile_seq, &amb, &tail, &ent, &tile_ent, &tile_cnt, &tile_off, &seg_start, &seg_cnt,
                          &chunk_first, &chunk_base, &cand_hash, &cand_pos, &segs, &tkey, &tcnt, &kept, &out_off,
                          &out_hash, &out_pos})
            b->release();
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    }
};

thread_local SummaryBuffers *tls_sum = nullptr;

DivTest make_div_test(uint64_t d) {
    DivTest t;
    t.shift = (uint32_t)__builtin_ctzll(d);
    const uint64_t d0 = d >> t.shift;
    uint64_t x = d0;  // correct to 3 bits for odd d0; each Newton step doubles them
    for (int i = 0; i < 5; ++i) x *= 2 - d0 * x;
    t.inv = x;
    t.limit = UINT64_MAX / d;
    t.pad = 0;
    return t;
}

uint64_t mix_hash_host(uint64_t v) {
    v ^= v >> 30;
    v *= 0xbf58476d1ce4e5b9ULL;
    v ^= v >> 27;
    v *= 0x94d049bb133111ebULL;
    v ^= v >> 31;
    return v;
}

// FNV-1a of the bytes finished by the selector's mix with the length (:570-579, :666).
uint64_t fingerprint_host(const char *s, int64_t len) {
    uint64_t h = 1469598103934665603ULL;
    for (int64_t i = 0; i < len; ++i) {
        h ^= (uint64_t)(unsigned char)s[i];
        h *= 1099511628211ULL;
    }
    return mix_hash_host(h ^ mix_hash_host((uint64_t)len));
}

}  // namespace
}  // namespace aw

using namespace aw;

// Candidates (and tables) of one chunk of sequences in device memory at most; the
// environment variable AW_SUMMARY_CHUNK_CANDIDATES overrides it (smaller chunks, more
// launches; the results do not depend on it).
static int64_t summary_chunk_candidates() {
    const char *e = getenv("AW_SUMMARY_CHUNK_CANDIDATES");
    const long long v = e ? atoll(e) : 0;
    return v > 0 ? (int64_t)v : ((int64_t)32 << 20);
}

extern "C" int aw_sequence_summary_batch(int n, const char *const *query, const int64_t *qlen,
                                         const char *const *reference, const int64_t *rlen,
                                         const uint64_t *modulos, aw_sequence_summary_t *out, int *identical,
                                         float *device_ms) {
    if (n < 0 || (n > 0 && (!query || !qlen || !reference || !rlen || !out || !identical))) {
        set_error("aw_sequence_summary_batch: invalid arguments");
        return AW_E_INVAL;
    }
    if (!tls_sum) {
        tls_sum = new SummaryBuffers();
        static thread_local struct Reaper {
            ~Reaper() { delete tls_sum; tls_sum = nullptr; }
        } reaper;
        (void)reaper;
    }
    SummaryBuffers &B = *tls_sum;
    B.sk_n = 0;
    if (device_ms) *device_ms = 0.f;
    if (n == 0) return AW_OK;
    const int nseq = 2 * n;
    std::vector<SeqDev> hs(nseq);
    int64_t total = 0, ntiles = 0;
    for (int i = 0; i < n; ++i) {
        if (qlen[i] < 0 || rlen[i] < 0 || (qlen[i] > 0 && !query[i]) || (rlen[i] > 0 && !reference[i]) ||
            std::max(qlen[i], rlen[i]) > (int64_t)UINT32_MAX) {
            set_error("aw_sequence_summary_batch: invalid pair");
            return AW_E_INVAL;
        }
        // sampling modulos of makeAlignmentSelectionPlan (:1752-1760) unless given
        uint64_t mod[3];
        const uint64_t mx = (uint64_t)std::max(qlen[i], rlen[i]);
        for (int sc = 0; sc < 3; ++sc) {
            if (modulos) mod[sc] = modulos[3 * (int64_t)i + sc];
            else {
                const uint64_t avail = mx >= kmer_len(sc) ? mx - kmer_len(sc) + 1 : 0;
                mod[sc] = std::max<uint64_t>(1, avail / SUM_TARGET[sc]);
            }
            if (mod[sc] == 0) {
                set_error("aw_sequence_summary_batch: sampling modulo 0");
                return AW_E_INVAL;
            }
        }
        for (int t = 0; t < 2; ++t) {
            SeqDev &S = hs[2 * i + t];
            S.off = total, S.len = t ? rlen[i] : qlen[i];
            for (int sc = 0; sc < 3; ++sc) S.div[sc] = make_div_test(mod[sc]);
            S.first_tile = (int32_t)ntiles;
            S.ntiles = (int32_t)((S.len + SUM_TILE - 1) / SUM_TILE);
            total += S.len, ntiles += S.ntiles;
        }
    }
    if (ntiles > INT32_MAX / 2) {
        set_error("aw_sequence_summary_batch: batch too large");
        return AW_E_INVAL;
    }
#define SCUDA(call)                                                                                   \
    do {                                                                                              \
        const cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                      \
            set_error((std::string("aw_sequence_summary_batch: ") + cudaGetErrorString(e_)).c_str()); \
            return AW_E_CUDA;                                                                         \
        }                                                                                             \
    } while (0)
    if (!B.st) SCUDA(cudaStreamCreateWithFlags(&B.st, cudaStreamNonBlocking));
    if (!B.e0) SCUDA(cudaEventCreate(&B.e0));
    if (!B.e1) SCUDA(cudaEventCreate(&B.e1));
    SCUDA(B.staging.ensure((size_t)total + 16));
    // host threads (one per 4 MB of bases, at most 8): the staging copy first, then the
    // fingerprints and identity flags while the device runs
    const int nth = (int)std::min<int64_t>(8, std::max<int64_t>(1, total >> 22));
    auto stage_work = [&](int w) {
        for (int i = w; i < n; i += nth) {
            if (qlen[i]) memcpy(B.staging.p + hs[2 * i].off, query[i], (size_t)qlen[i]);
            if (rlen[i]) memcpy(B.staging.p + hs[2 * i + 1].off, reference[i], (size_t)rlen[i]);
        }
    };
    {
        std::vector<std::thread> sth;
        for (int w = 1; w < nth; ++w) sth.emplace_back(stage_work, w);
        stage_work(0);
        for (auto &x : sth) x.join();
    }
    std::vector<uint64_t> fp(nseq);
    std::vector<std::thread> fth;
    auto fp_work = [&](int w) {
        for (int j = w; j < nseq; j += nth) {
            const int i = j >> 1;
            fp[j] = (j & 1) ? fingerprint_host(reference[i], rlen[i]) : fingerprint_host(query[i], qlen[i]);
            if (!(j & 1))
                identical[i] = qlen[i] == rlen[i] && (qlen[i] == 0 || memcmp(query[i], reference[i], (size_t)qlen[i]) == 0);
        }
    };
    for (int w = 1; w < nth; ++w) fth.emplace_back(fp_work, w);
    struct Joiner {
        std::vector<std::thread> &t;
        ~Joiner() {
            for (auto &x : t)
                if (x.joinable()) x.join();
        }
    } joiner{fth};
    std::vector<int32_t> tseq((size_t)std::max<int64_t>(ntiles, 1));
    for (int j = 0; j < nseq; ++j)
        for (int32_t k = 0; k < hs[j].ntiles; ++k) tseq[(size_t)hs[j].first_tile + k] = j;
    SCUDA(B.bases.ensure((size_t)total + 16));
    SCUDA(B.seqs.ensure(sizeof(SeqDev) * (size_t)nseq));
    SCUDA(B.tile_seq.ensure(4 * tseq.size()));
    SCUDA(B.amb.ensure(8 * (size_t)nseq));
    SCUDA(B.tail.ensure(8 * (size_t)nseq));
    SCUDA(B.ent.ensure(8 * (size_t)nseq));
    SCUDA(B.tile_ent.ensure(8 * (size_t)std::max<int64_t>(ntiles, 1)));
    SCUDA(B.tile_cnt.ensure(4 * 3 * (size_t)std::max<int64_t>(ntiles, 1)));
    SCUDA(B.tile_off.ensure(8 * 3 * (size_t)(ntiles + 1)));
    SCUDA(B.seg_start.ensure(8 * 3 * (size_t)nseq));
    SCUDA(B.seg_cnt.ensure(8 * 3 * (size_t)nseq));
    cudaStream_t st = B.st;
    float ms_total = 0.f;
    SCUDA(cudaEventRecord(B.e0, st));
    if (total) SCUDA(cudaMemcpyAsync(B.bases.p, B.staging.p, (size_t)total, cudaMemcpyHostToDevice, st));
    SCUDA(cudaMemcpyAsync(B.seqs.p, hs.data(), sizeof(SeqDev) * (size_t)nseq, cudaMemcpyHostToDevice, st));
    SCUDA(cudaMemcpyAsync(B.tile_seq.p, tseq.data(), 4 * tseq.size(), cudaMemcpyHostToDevice, st));
    SCUDA(cudaMemsetAsync(B.amb.p, 0, 8 * (size_t)nseq, st));
    SCUDA(cudaMemsetAsync(B.tail.p, 0, 8 * (size_t)nseq, st));
    SCUDA(cudaMemsetAsync(B.tile_cnt.p, 0, 4 * 3 * (size_t)std::max<int64_t>(ntiles, 1), st));
    // 1. count pass (tiles in launches of at most 2^30 CTAs)
    for (int64_t t0 = 0; t0 < ntiles; t0 += (int64_t)1 << 30) {
        const int64_t nt = std::min<int64_t>(ntiles - t0, (int64_t)1 << 30);
        summary_tile_kernel<true><<<(unsigned)nt, SUM_THREADS, 0, st>>>(
            B.bases.as<uint8_t>(), B.seqs.as<SeqDev>(), B.tile_seq.as<int32_t>(), (int32_t)t0, ntiles,
            B.amb.as<unsigned long long>(), B.tail.as<unsigned long long>(), B.tile_ent.as<double>(),
            B.tile_cnt.as<uint32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr);
        SCUDA(cudaGetLastError());
    }
    // 2. ranks of the tiles' candidates per scale, ranges per (sequence, scale)
    scan_rows_kernel<<<3, 1024, 0, st>>>(B.tile_cnt.as<uint32_t>(), B.tile_off.as<int64_t>(), ntiles);
    SCUDA(cudaGetLastError());
    segments_kernel<<<(nseq + 255) / 256, 256, 0, st>>>(B.seqs.as<SeqDev>(), nseq, B.tile_off.as<int64_t>(), ntiles,
                                                         B.seg_start.as<int64_t>(), B.seg_cnt.as<int64_t>(),
                                                         B.tile_ent.as<double>(), B.ent.as<double>());
    SCUDA(cudaGetLastError());
    std::vector<unsigned long long> hamb(nseq), htail(nseq);
    std::vector<double> hent(nseq);
    std::vector<int64_t> sstart(3 * (size_t)nseq), scnt(3 * (size_t)nseq);
    SCUDA(cudaMemcpyAsync(hamb.data(), B.amb.p, 8 * (size_t)nseq, cudaMemcpyDeviceToHost, st));
    SCUDA(cudaMemcpyAsync(htail.data(), B.tail.p, 8 * (size_t)nseq, cudaMemcpyDeviceToHost, st));
    SCUDA(cudaMemcpyAsync(hent.data(), B.ent.p, 8 * (size_t)nseq, cudaMemcpyDeviceToHost, st));
    SCUDA(cudaMemcpyAsync(sstart.data(), B.seg_start.p, 8 * sstart.size(), cudaMemcpyDeviceToHost, st));
    SCUDA(cudaMemcpyAsync(scnt.data(), B.seg_cnt.p, 8 * scnt.size(), cudaMemcpyDeviceToHost, st));
    SCUDA(cudaEventRecord(B.e1, st));
    SCUDA(cudaStreamSynchronize(st));
    {
        float ms = 0.f;
        SCUDA(cudaEventElapsedTime(&ms, B.e0, B.e1));
        ms_total += ms;
    }
    // the kept entries are at most the candidates: one page-locked output of that size
    int64_t all_cands = 0;
    for (int64_t c : scnt) all_cands += c;
    SCUDA(B.sk_hash.ensure(8 * (size_t)all_cands + 8));
    SCUDA(B.sk_pos.ensure(4 * (size_t)all_cands + 4));
    // 3-5. chunks of whole sequences (a query and its reference together is not needed:
    // the sketches are per sequence)
    int64_t out_total = 0;
    const int64_t chunk_budget = summary_chunk_candidates();
    std::vector<int64_t> sk_off(3 * (size_t)nseq, 0);
    for (int j0 = 0; j0 < nseq;) {
        int j1 = j0;
        int64_t cands = 0;
        while (j1 < nseq) {
            const int64_t c = scnt[3 * (size_t)j1] + scnt[3 * (size_t)j1 + 1] + scnt[3 * (size_t)j1 + 2];
            if (j1 > j0 && cands + c > chunk_budget) break;
            cands += c, ++j1;
        }
        const int nsg = 3 * (j1 - j0);
        // chunk layout: scale regions of candidates back to back; a table per segment
        int64_t first[3], base[3], acc = 0;
        for (int sc = 0; sc < 3; ++sc) {
            first[sc] = sstart[3 * (size_t)j0 + sc];
            base[sc] = acc;
            const int64_t last = j1 < nseq ? sstart[3 * (size_t)j1 + sc] : sstart[3 * (size_t)(j1 - 1) + sc] + scnt[3 * (size_t)(j1 - 1) + sc];
            acc += last - first[sc];
        }
        std::vector<SegDev> hsg(nsg);
        int64_t tslots = 0;
        for (int j = j0; j < j1; ++j)
            for (int sc = 0; sc < 3; ++sc) {
                SegDev &G = hsg[3 * (j - j0) + sc];
                G.cand = base[sc] + (sstart[3 * (size_t)j + sc] - first[sc]);
                G.count = scnt[3 * (size_t)j + sc];
                int64_t ts = 64;
                while (ts < 2 * G.count) ts <<= 1;
                G.table = tslots, G.tsize = ts;
                tslots += ts;
            }
        SCUDA(B.chunk_first.ensure(64));
        SCUDA(B.chunk_base.ensure(64));
        SCUDA(B.cand_hash.ensure(8 * (size_t)std::max<int64_t>(acc, 1)));
        SCUDA(B.cand_pos.ensure(4 * (size_t)std::max<int64_t>(acc, 1)));
        SCUDA(B.segs.ensure(sizeof(SegDev) * (size_t)nsg));
        SCUDA(B.tkey.ensure(8 * (size_t)tslots));
        SCUDA(B.tcnt.ensure(4 * (size_t)tslots));
        SCUDA(B.kept.ensure(4 * (size_t)nsg));
        SCUDA(B.out_off.ensure(8 * (size_t)(nsg + 1)));
        SCUDA(B.out_hash.ensure(8 * (size_t)std::max<int64_t>(acc, 1)));
        SCUDA(B.out_pos.ensure(4 * (size_t)std::max<int64_t>(acc, 1)));
        SCUDA(cudaMemcpyAsync(B.chunk_first.p, first, sizeof(first), cudaMemcpyHostToDevice, st));
        SCUDA(cudaMemcpyAsync(B.chunk_base.p, base, sizeof(base), cudaMemcpyHostToDevice, st));
        SCUDA(cudaMemcpyAsync(B.segs.p, hsg.data(), sizeof(SegDev) * (size_t)nsg, cudaMemcpyHostToDevice, st));
        SCUDA(cudaEventRecord(B.e0, st));
        SCUDA(cudaMemsetAsync(B.tcnt.p, 0, 4 * (size_t)tslots, st));
        const int32_t t0 = hs[j0].first_tile;
        const int64_t nt = (int64_t)hs[j1 - 1].first_tile + hs[j1 - 1].ntiles - t0;
        if (nt > 0) {
            summary_tile_kernel<false><<<(unsigned)nt, SUM_THREADS, 0, st>>>(
                B.bases.as<uint8_t>(), B.seqs.as<SeqDev>(), B.tile_seq.as<int32_t>(), t0, ntiles, nullptr, nullptr,
                nullptr, nullptr, B.tile_off.as<int64_t>(), B.chunk_first.as<int64_t>(), B.chunk_base.as<int64_t>(),
                B.cand_hash.as<uint64_t>(), B.cand_pos.as<uint32_t>());
            SCUDA(cudaGetLastError());
        }
        cap_kernel<<<(nsg + 7) / 8, 256, 0, st>>>(B.segs.as<SegDev>(), nsg, B.cand_hash.as<uint64_t>(),
                                                  B.cand_pos.as<uint32_t>(), B.tkey.as<unsigned long long>(),
                                                  B.tcnt.as<uint32_t>(), B.kept.as<uint32_t>());
        SCUDA(cudaGetLastError());
        scan_rows_kernel<<<1, 1024, 0, st>>>(B.kept.as<uint32_t>(), B.out_off.as<int64_t>(), nsg);
        SCUDA(cudaGetLastError());
        gather_kernel<<<(nsg + 7) / 8, 256, 0, st>>>(B.segs.as<SegDev>(), nsg, B.out_off.as<int64_t>(),
                                                     B.cand_hash.as<uint64_t>(), B.cand_pos.as<uint32_t>(),
                                                     B.kept.as<uint32_t>(), B.out_hash.as<uint64_t>(),
                                                     B.out_pos.as<uint32_t>());
        SCUDA(cudaGetLastError());
        SCUDA(cudaEventRecord(B.e1, st));
        std::vector<int64_t> hoff((size_t)nsg + 1);
        SCUDA(cudaMemcpyAsync(hoff.data(), B.out_off.p, 8 * hoff.size(), cudaMemcpyDeviceToHost, st));
        SCUDA(cudaStreamSynchronize(st));
        {
            float ms = 0.f;
            SCUDA(cudaEventElapsedTime(&ms, B.e0, B.e1));
            ms_total += ms;
        }
        const int64_t kept_total = hoff[(size_t)nsg];
        if (kept_total) {
            SCUDA(cudaMemcpyAsync(B.sk_hash.as<uint64_t>() + out_total, B.out_hash.p, 8 * (size_t)kept_total,
                                  cudaMemcpyDeviceToHost, st));
            SCUDA(cudaMemcpyAsync(B.sk_pos.as<uint32_t>() + out_total, B.out_pos.p, 4 * (size_t)kept_total,
                                  cudaMemcpyDeviceToHost, st));
            SCUDA(cudaStreamSynchronize(st));
        }
        for (int g = 0; g < nsg; ++g) {
            sk_off[3 * (size_t)j0 + g] = out_total + hoff[(size_t)g];
            scnt[3 * (size_t)j0 + g] = hoff[(size_t)g + 1] - hoff[(size_t)g];
        }
        out_total += kept_total;
        j0 = j1;
    }
    B.sk_n = out_total;
    if (device_ms) *device_ms = ms_total;
    fp_work(0);
    for (auto &x : fth) x.join();
    for (int j = 0; j < nseq; ++j) {
        aw_sequence_summary_t &o = out[j];
        const int64_t len = hs[j].len;
        o.fingerprint = fp[j];
        o.ambiguous_fraction = len ? (double)hamb[j] / (double)len : 0.0;
        o.low_complexity_fraction = len ? (double)htail[j] / (double)len : 0.0;
        o.normalized_entropy = len ? hent[j] / (double)len : 0.0;
        for (int sc = 0; sc < 3; ++sc) {
            o.sketch_offset[sc] = sk_off[3 * (size_t)j + sc];
            o.sketch_count[sc] = scnt[3 * (size_t)j + sc];
        }
    }
    return AW_OK;
#undef SCUDA
}

extern "C" int64_t aw_sequence_summary_sketches(uint64_t *hash, uint32_t *position, int64_t capacity) {
    if (!tls_sum) return 0;
    const int64_t n = tls_sum->sk_n;
    if (!hash && !position) return n;
    if (capacity < n || !hash || !position) {
        set_error("aw_sequence_summary_sketches: capacity below the number of entries");
        return AW_E_INVAL;
    }
    if (n) {
        memcpy(hash, tls_sum->sk_hash.p, 8 * (size_t)n);
        memcpy(position, tls_sum->sk_pos.p, 4 * (size_t)n);
    }
    return n;
}

extern "C" int64_t aw_sequence_summary_sketch_view(const uint64_t **hash, const uint32_t **position) {
    if (!tls_sum || !hash || !position) return tls_sum ? tls_sum->sk_n : 0;
    *hash = tls_sum->sk_hash.as<uint64_t>();
    *position = tls_sum->sk_pos.as<uint32_t>();
    return tls_sum->sk_n;
}
