// Internal types shared by the KSW2 / WFA kernels and the C-ABI host layer.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include <algorithm>

#define AW_NEG_INF (-0x40000000)
#define AW_E_CUDA_INTERNAL (-2)
#define AW_E_NOMEM_INTERNAL (-3)

// Flags of ksw_extd2 (minimap2/ksw2.h:20-34).
#define AW_EZ_SCORE_ONLY     0x01
#define AW_EZ_RIGHT          0x02
#define AW_EZ_GENERIC_SC     0x04
#define AW_EZ_APPROX_MAX     0x08
#define AW_EZ_APPROX_DROP    0x10
#define AW_EZ_EXTZ_ONLY      0x40
#define AW_EZ_REV_CIGAR      0x80
#define AW_EZ_SPLICE_MASK    0x700
#define AW_EZ_SEMIGLOBAL_END 0x800
#define AW_EZ_SINGLETRACK    0x1000
// with AW_EZ_SINGLETRACK: ksw_extd2_singletrack_sse (16-byte blocks and its end rules)
#define AW_EZ_SSE_SINGLETRACK 0x4000

namespace aw {

// Per-launch scoring constants, after the q+e <= q2+e2 swap of
// minimap2/ksw2_extd2_sse.c:83.
struct KswScore {
    int q, e, q2, e2;
    int qe, qe2;
    int qe_pre;               // q+e of the caller's argument order: seeds H (ksw2_extd2_sse.c:73, :367)
    int mch;                  // mat[0], the clamp of ksw2_extd2_sse.c:252
    int long_thres, long_diff;  // ksw2_extd2_sse.c:107-110
    uint32_t tab_lo[8];       // score row per target code: bytes for query codes 0..3
    uint32_t tab_hi[8];       //                             bytes for query codes 4..7
};

// One pair of the batch as the kernels see it.
struct KswPair {
    int64_t qoff, toff;   // byte offsets of the 0..m-1 codes in the sequence arenas
    int64_t tb_off;       // byte offset of this pair's traceback (CIGAR modes)
    int64_t bnd_off;      // word offset of this pair's strip-boundary columns
    int64_t cig_off;      // word offset of this pair's CIGAR slot (capacity qlen+tlen)
    int32_t qlen, tlen;
};

// Scalar ksw_extz_t fields produced on the device (minimap2/ksw2.h:40-50).
struct KswOut {
    int32_t score, max, max_q, max_t, mqe, mqe_t, mte, mte_q;
    int32_t n_cigar, zdropped, reach_end, stopped;
};

struct KswFullArgs {
    const uint8_t *qcodes, *tcodes;
    const KswPair *pairs;
    const int32_t *order;     // processing order (largest first)
    int32_t n;
    uint8_t *tb;              // traceback arena (CIGAR modes)
    uint32_t *bnd;            // strip-boundary arena
    KswOut *out;
    int32_t *queue;           // work-queue head (device counter)
    int32_t *error;           // set non-zero if a bounded wait gave up
    KswScore sc;
    // the calling thread's deadline (globaltimer ns) or null: pairs still running when it
    // passes stop with ez->stopped = 1 (the cooperative stop of minimap2/ksw2_progress.c)
    const unsigned long long *deadline = nullptr;
    // 1, passed at run time: the strip kernel's 2-input adds are multiply-adds by it, which
    // the compiler keeps on the FMA pipe
    uint32_t one = 1;
};

#ifdef __CUDACC__
__device__ __forceinline__ bool aw_deadline_passed(const unsigned long long *d) {
    if (!d) return false;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t >= *(const volatile unsigned long long *)d;
}
#endif

// Traceback geometry of the full-matrix strip kernel: strips of KSW_STRIP = 512 target
// columns in KSW_GROUPS = 64 groups of KSW_COLS = 8; a step of a strip stores one
// KSW_COLS-byte word per group, the word of group g at row r being stored at step r + g:
// byte ((strip * (qlen + KSW_LAG) + r + g) * KSW_GROUPS + g) * KSW_COLS + (col & 7).
constexpr int KSW_COLS = 8;
constexpr int KSW_GROUPS = 64;
constexpr int KSW_STRIP = KSW_GROUPS * KSW_COLS;
constexpr int KSW_LAG = KSW_GROUPS - 1;

inline int64_t ksw_full_tb_bytes(int qlen, int tlen) {
    const int64_t nstrip = (tlen + KSW_STRIP - 1) / KSW_STRIP;
    return nstrip * (int64_t)(qlen + KSW_LAG) * KSW_STRIP;
}
// boundary column of a strip: one 8-byte entry per row and one for the strip's last-row H
inline int64_t ksw_full_bnd_words(int qlen, int tlen) {
    const int64_t nstrip = (tlen + KSW_STRIP - 1) / KSW_STRIP;
    return nstrip * ((int64_t)qlen + 1) * 2;
}

// Grow-only device allocation (pooled per host thread or per plan).
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    // Grows by half the current capacity, at most 256 MiB more than that (pooled buffers
    // see batches of varying size, and every cudaFree synchronises the device), falling
    // back to exactly n when the larger request does not fit.
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        const size_t grown = cap + std::min(cap / 2, (size_t)256 << 20);
        if (p) cudaFree(p);
        p = nullptr;
        size_t want = n < 4096 ? 4096 : n;
        if (grown > want && cap > 0) {
            if (cudaMalloc(&p, grown) == cudaSuccess) {
                cap = grown;
                return cudaSuccess;
            }
            cudaGetLastError();
        }
        cap = 0;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr, cap = 0;
    }
    template <class T> T *as() const { return (T *)p; }
};

void set_error(const char *msg);

// Traceback budget of the calling thread's batches, 0 = process-wide (ksw2_api.cu).
void set_thread_tb_budget(int64_t bytes);
// Allocates the calling thread's pooled traceback arena (ksw2_api.cu).
int reserve_thread_tb(int64_t bytes);

// Strip-path parameter check + score table (ksw2_api.cu).
int full_path_params(int qlen, int tlen, int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2,
                     int8_t e2, int flag, KswScore *S);

// Launchers (ksw2_full.cu).
int ksw_full_occupancy(int flag, int warps_per_pair, int groups_per_cta);
cudaError_t launch_ksw_full(const KswFullArgs &a, int flag, int warps_per_pair,
                            int groups_per_cta, int ctas, cudaStream_t st);
cudaError_t launch_ksw_backtrack_full(const KswPair *pairs, const int32_t *order, int n,
                                      const uint8_t *tb, KswOut *out, uint32_t *cig,
                                      int flag, cudaStream_t st);
// Writes globaltimer + remaining_ns (or "never" for ~0) to *deadline on the stream, so
// the deadline counts from when the stream reaches this call.
cudaError_t launch_set_deadline(unsigned long long *deadline, unsigned long long remaining_ns, cudaStream_t st);
cudaError_t launch_ksw_pack_cigar(const KswPair *pairs, int n, const KswOut *out,
                                  const uint32_t *cig, const int64_t *packed_off,
                                  uint32_t *packed, cudaStream_t st);

}  // namespace aw
