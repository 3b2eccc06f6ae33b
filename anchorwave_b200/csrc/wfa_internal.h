// Internal types of the WFA kernel (wfa.cu) and its host layer (wfa_api.cu).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace aw {

// WF status codes (WFA2-lib wavefront/wfa.h:46-55) plus internal retry/overflow.
constexpr int WFA_COMPLETED = 0;
constexpr int WFA_OOM = -200;
constexpr int WFA_UNATTAINABLE = -300;
constexpr int WFA_RETRY = -1000;     // device pool exhausted: re-run in a later round
constexpr int WFA_OVERFLOW = -1001;  // a per-pair bound was exceeded
constexpr int WFA_WIDE = -1002;      // wavefront wider than a warp's share: re-run by the cluster kernel

struct WfaPen {
    int x, o1, e1, o2, e2;
};

struct WfaPairDev {
    int64_t poff, toff;    // padded pattern / text in the sequence arenas (8-byte aligned)
    int32_t plen, tlen;
    int64_t ops_off;       // CIGAR operation slot (plen + tlen + 8 chars)
    int64_t ctab_off;      // header-chunk table (int64 pool offsets), ctab_cap entries
    int32_t ctab_cap;
    int32_t packed;        // 1: pattern and text are uppercase ACGT only (set on the device)
};

struct WfaOutDev {
    int32_t status, score, n_ops, final_s;
    int64_t mem_bytes;
};

struct WfaArgs {
    const uint8_t *pat, *txt;
    const uint64_t *ppat, *ptxt;  // the same arenas at 2 bits per base (32 bases per word)
    const WfaPairDev *pairs;
    const int32_t *order;
    int32_t n;
    const int32_t *order_long;  // pairs each run on a whole CTA first (high memory), n_long of them
    int32_t n_long;
    uint8_t *pool;
    int64_t pool_bytes;
    unsigned long long *pool_head;
    int64_t *ctab;
    char *ops;
    WfaOutDev *out;
    int32_t *queue;       // [0] next position of `order`, [1] pairs running on warps,
                          // [2] next position of `order_long`
    WfaPen pen;
    int singletrack;
    int piggyback;        // medium / low memory: ring of recent scores + packed-CIGAR blocks
    int max_score_scope;
    int wide_width;       // warp kernel: a pair whose wavefront grows wider stops with WFA_WIDE (0 = never)
    int wide_width_tail;  // the same once every pair has started and at most wide_tail_pairs
    int wide_tail_pairs;  // still run on warps (<= wide_width)
    int wide_width_cta;   // a pair on a whole CTA whose wavefront grows wider stops with WFA_WIDE
};

cudaError_t launch_wfa(const WfaArgs &a, int ctas, cudaStream_t st);
// The cluster kernel (high memory: standard and Singletrack): one cluster of `cl` CTAs per
// pair, the diagonals of a wavefront spread over all of its threads; `clusters` clusters
// take the pairs of a.order in turn.
cudaError_t launch_wfa_wide(const WfaArgs &a, int clusters, int cl, cudaStream_t st);
// Clusters of `cl` CTAs of the cluster kernel that fit on the device at once for a score
// scope (0 if none, or if the scope is too large for the kernel's header ring).
int wfa_wide_clusters(int cl, int scope);
// 2-bit copies of the pattern and text arenas (A=0, C=1, G=2, T=3, any other byte 0), and
// the per-pair flag that the pair's sequences are uppercase ACGT only.
cudaError_t launch_wfa_pack(const uint8_t *pat, int64_t pbytes, uint64_t *ppat, const uint8_t *txt, int64_t tbytes,
                            uint64_t *ptxt, WfaPairDev *pairs, int n, cudaStream_t st);
int wfa_occupancy(bool piggyback);

}  // namespace aw
