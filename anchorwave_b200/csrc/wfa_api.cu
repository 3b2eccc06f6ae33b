// C-ABI host layer of the WFA kernel: a GPU aligner handle that mirrors
// wavefront_aligner_new / wavefront_align / wavefront_aligner_delete
// (WFA2-lib wavefront/wfa.h:129-134, :210-215) with the attributes AnchorWave sets
// (src/myImportandFunction/WfaAlignment.cpp:143-170), plus a batched entry.
// One handle per host thread (AnchorWave keeps a thread-local aligner per memory
// mode, WfaAlignment.cpp:217-221); each handle owns a stream and pooled buffers.
#include "aw_internal.h"
#include "wfa_internal.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace aw;

namespace {

constexpr int HDR_CHUNK = 256;
constexpr int PAD = 16;  // sentinel bytes after every sequence

struct PinBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr, cap = 0;
        const size_t want = std::max(n + n / 2, (size_t)4096);
        const cudaError_t e = cudaMallocHost(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    ~PinBuf() {
        if (p) cudaFreeHost(p);
    }
};

int64_t al8(int64_t v) { return (v + 7) & ~(int64_t)7; }

// Wavefront width from which a warp hands its pair to the cluster kernel, and the CTAs of a
// cluster (aw_set_wfa_wide).
std::atomic<int> g_wide_width{8192};
std::atomic<int> g_wide_tail{1024};
std::atomic<int> g_wide_cluster{8};
// Pairs with pattern + text length from which a pair runs on a whole CTA (aw_set_wfa_long).
std::atomic<int> g_long_sum{1536};

}  // namespace

struct wavefront_aligner_gpu {
    wavefront_gpu_attr_t attr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DevBuf d_pat, d_txt, d_pairs, d_order, d_pool, d_head, d_ctab, d_ops, d_out, d_queue;
    DevBuf d_ppat, d_ptxt;  // 2-bit copies of the sequence arenas
    PinBuf h_pat, h_txt, h_ops;
    std::vector<WfaPairDev> pairs;
    std::vector<WfaOutDev> outs;
    // single-call result
    std::string ops;
    int score = 0;
    int64_t mem_pair_max = 0, mem_total = 0;
    int sms = 0;
    float last_ms = 0.f;
    int last_launches = 0;
    int last_cluster_launches = 0, last_cluster_pairs = 0;
    ~wavefront_aligner_gpu() {
        d_pat.release(), d_txt.release(), d_pairs.release(), d_order.release(), d_pool.release();
        d_head.release(), d_ctab.release(), d_ops.release(), d_out.release(), d_queue.release();
        d_ppat.release(), d_ptxt.release();
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    }
};

#define WCUDA(call)                                                         \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) {                                            \
            set_error((std::string(#call) + ": " + cudaGetErrorString(_e)).c_str()); \
            return AW_E_CUDA;                                               \
        }                                                                   \
    } while (0)

static int run_batch(wavefront_aligner_gpu *al, int n, const char *const *pattern, const int *plen,
                     const char *const *text, const int *tlen) {
    const wavefront_gpu_attr_t &A = al->attr;
    al->pairs.assign(n, WfaPairDev{});
    al->outs.assign(n, WfaOutDev{});
    int64_t pb = 0, tb = 0, ob = 0, cb = 0;
    for (int i = 0; i < n; ++i) {
        WfaPairDev &P = al->pairs[i];
        const int p = plen[i], t = tlen[i];
        P.plen = p, P.tlen = t;
        P.poff = pb, P.toff = tb;
        pb += al8(p + PAD) + 8, tb += al8(t + PAD) + 8;
        P.ops_off = ob;
        ob += (int64_t)p + t + 8;
        // score bound: all mismatches plus one gap for the length difference
        // (wavefront/wavefront_components.c:118-124)
        const int64_t d = std::abs(p - t);
        const int64_t bound = (int64_t)std::min(p, t) * A.mismatch +
                              std::max(A.gap_opening1 + d * A.gap_extension1, A.gap_opening2 + d * A.gap_extension2) + 2;
        P.ctab_cap = (int32_t)((bound + HDR_CHUNK) / HDR_CHUNK + 1);
        P.ctab_off = cb;
        cb += P.ctab_cap;
    }
    WCUDA(al->h_pat.ensure((size_t)pb + 64));
    WCUDA(al->h_txt.ensure((size_t)tb + 64));
    uint8_t *hp = (uint8_t *)al->h_pat.p, *ht = (uint8_t *)al->h_txt.p;
    for (int i = 0; i < n; ++i) {
        const WfaPairDev &P = al->pairs[i];
        if (P.plen > 0) memcpy(hp + P.poff, pattern[i], (size_t)P.plen);
        memset(hp + P.poff + P.plen, '!', (size_t)(al8(P.plen + PAD) + 8 - P.plen));
        if (P.tlen > 0) memcpy(ht + P.toff, text[i], (size_t)P.tlen);
        memset(ht + P.toff + P.tlen, '?', (size_t)(al8(P.tlen + PAD) + 8 - P.tlen));
    }
    std::vector<int32_t> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const int64_t la = (int64_t)plen[a] + tlen[a], lb = (int64_t)plen[b] + tlen[b];
        return la != lb ? la > lb : a < b;
    });
    WCUDA(al->d_pat.ensure((size_t)pb + 64));
    WCUDA(al->d_txt.ensure((size_t)tb + 64));
    WCUDA(al->d_ppat.ensure(8 * (size_t)((pb + 31) / 32 + 2)));
    WCUDA(al->d_ptxt.ensure(8 * (size_t)((tb + 31) / 32 + 2)));
    WCUDA(al->d_pairs.ensure(sizeof(WfaPairDev) * (size_t)n));
    WCUDA(al->d_order.ensure(sizeof(int32_t) * (size_t)n));
    WCUDA(al->d_ctab.ensure(8 * (size_t)cb + 64));
    WCUDA(al->d_ops.ensure((size_t)ob + 64));
    WCUDA(al->d_out.ensure(sizeof(WfaOutDev) * (size_t)n));
    WCUDA(al->d_queue.ensure(64));
    WCUDA(al->d_head.ensure(64));
    // device pool: 85% of free memory (capped by max_memory_abort when set)
    if (al->d_pool.cap == 0) {
        size_t fr = 0, tot = 0;
        WCUDA(cudaMemGetInfo(&fr, &tot));
        int64_t want = (int64_t)(fr * 0.85);
        if (A.max_memory_abort > 0) want = std::min<int64_t>(want, A.max_memory_abort);
        // piggyback blocks are addressed by 32-bit indices of 8-byte units
        if (A.memory_mode != 0) want = std::min<int64_t>(want, ((int64_t)1 << 35) - ((int64_t)1 << 20));
        want = std::max<int64_t>(want, (int64_t)64 << 20);
        WCUDA(al->d_pool.ensure((size_t)want));
    }
    WCUDA(cudaMemcpyAsync(al->d_pat.p, hp, (size_t)pb, cudaMemcpyHostToDevice, al->st));
    WCUDA(cudaMemcpyAsync(al->d_txt.p, ht, (size_t)tb, cudaMemcpyHostToDevice, al->st));
    WCUDA(cudaMemcpyAsync(al->d_pairs.p, al->pairs.data(), sizeof(WfaPairDev) * (size_t)n, cudaMemcpyHostToDevice,
                          al->st));
    // 2-bit arenas for the extend step, and which pairs may use them
    WCUDA(launch_wfa_pack(al->d_pat.as<uint8_t>(), pb, al->d_ppat.as<uint64_t>(), al->d_txt.as<uint8_t>(), tb,
                          al->d_ptxt.as<uint64_t>(), al->d_pairs.as<WfaPairDev>(), n, al->st));
    WfaArgs W;
    W.pat = al->d_pat.as<uint8_t>(), W.txt = al->d_txt.as<uint8_t>();
    W.ppat = al->d_ppat.as<uint64_t>(), W.ptxt = al->d_ptxt.as<uint64_t>();
    W.pairs = al->d_pairs.as<WfaPairDev>();
    W.pool = al->d_pool.as<uint8_t>(), W.pool_bytes = (int64_t)al->d_pool.cap;
    W.pool_head = al->d_head.as<unsigned long long>();
    W.ctab = al->d_ctab.as<int64_t>();
    W.ops = al->d_ops.as<char>();
    W.out = al->d_out.as<WfaOutDev>();
    W.queue = al->d_queue.as<int32_t>();
    W.pen = WfaPen{A.mismatch, A.gap_opening1, A.gap_extension1, A.gap_opening2, A.gap_extension2};
    W.piggyback = A.memory_mode != 0 ? 1 : 0;
    W.singletrack = A.singletrack && !W.piggyback ? 1 : 0;
    const int scope = std::max(A.gap_opening1 + A.gap_extension1, A.gap_opening2 + A.gap_extension2);
    W.max_score_scope = std::max(scope, A.mismatch) + 1;
    const int occ = std::max(1, wfa_occupancy(W.piggyback != 0));
    // Pairs whose wavefront outgrows a warp (high memory only) stop with WFA_WIDE and run
    // again, from score 0, on the cluster kernel once the warp phase is over.
    const int cl = std::min(8, std::max(1, g_wide_cluster.load()));
    const int wide_clusters = W.piggyback ? 0 : wfa_wide_clusters(cl, W.max_score_scope);
    W.wide_width = wide_clusters > 0 ? std::max(0, g_wide_width.load()) : 0;
    W.wide_width_tail = std::min(W.wide_width, std::max(0, g_wide_tail.load()));
    W.wide_tail_pairs = std::max(1, wide_clusters);
    W.wide_width_cta = W.wide_width;
    const int64_t long_sum = g_long_sum.load();
    std::vector<int32_t> staged;
    // Rounds: every round restarts the pool and runs up to `chunk` pending pairs, largest
    // first; pairs that found the pool exhausted stay pending.  A round that completes
    // nothing halves the chunk (the pairs in flight together share the pool), one that
    // completes all of its pairs doubles it again; a pair that cannot finish with the whole
    // pool to itself reports WF_STATUS_OOM (the reference's max-memory abort).
    std::vector<int32_t> wide;
    al->last_cluster_launches = 0;
    float total_ms = 0.f;
    int launches = 0;
    for (int phase = 0; phase < 2; ++phase) {
        std::vector<int32_t> pending = phase == 0 ? order : wide;
        size_t chunk = pending.size();
        while (!pending.empty()) {
            const size_t take = std::min(chunk, pending.size());
            std::vector<int32_t> batch(pending.begin(), pending.begin() + (std::ptrdiff_t)take);
            // warp phase: the long pairs (still largest first) ahead of the others, each taken by
            // a whole CTA before the CTAs' warps take the others one each
            int32_t n_long = 0;
            staged.clear();
            if (phase == 0 && long_sum > 0) {
                for (int32_t i : batch)
                    if ((int64_t)plen[i] + tlen[i] >= long_sum) staged.push_back(i);
                n_long = (int32_t)staged.size();
                for (int32_t i : batch)
                    if ((int64_t)plen[i] + tlen[i] < long_sum) staged.push_back(i);
            } else {
                staged = batch;
            }
            WCUDA(cudaMemcpyAsync(al->d_order.p, staged.data(), sizeof(int32_t) * staged.size(), cudaMemcpyHostToDevice,
                                  al->st));
            WCUDA(cudaMemsetAsync(al->d_queue.p, 0, 16, al->st));
            WCUDA(cudaMemsetAsync(al->d_head.p, 0, 8, al->st));
            W.order_long = al->d_order.as<int32_t>();
            W.n_long = n_long;
            W.order = al->d_order.as<int32_t>() + n_long;
            W.n = (int32_t)staged.size() - n_long;
            WCUDA(cudaEventRecord(al->e0, al->st));
            if (phase == 0) {
                const int ctas = std::max(1, std::min(std::max((W.n + 3) / 4, W.n_long), occ * al->sms));
                WCUDA(launch_wfa(W, ctas, al->st));
            } else {
                ++al->last_cluster_launches;
                WCUDA(launch_wfa_wide(W, std::min(W.n, wide_clusters), cl, al->st));
            }
            WCUDA(cudaEventRecord(al->e1, al->st));
            ++launches;
            WCUDA(cudaMemcpyAsync(al->outs.data(), al->d_out.p, sizeof(WfaOutDev) * (size_t)n, cudaMemcpyDeviceToHost,
                                  al->st));
            WCUDA(cudaStreamSynchronize(al->st));
            float ms = 0.f;
            WCUDA(cudaEventElapsedTime(&ms, al->e0, al->e1));
            total_ms += ms;
            std::vector<int32_t> again;
            size_t handed = 0;
            for (int32_t i : batch) {
                if (al->outs[i].status == WFA_RETRY) again.push_back(i);
                if (al->outs[i].status == WFA_WIDE) wide.push_back(i), ++handed;
            }
            if (getenv("AW_VERBOSE"))
                fprintf(stderr, "[aw_b200] WFA round %d (%s): %zu pairs, %zu to retry, %zu to the cluster kernel, %.1f ms\n",
                        launches, phase ? "cluster" : "warp", batch.size(), again.size(), handed, ms);
            const size_t done = batch.size() - again.size();
            if (done == 0 && take == 1) {
                al->outs[batch[0]].status = WFA_OOM;
                again.clear();
            } else if (done == 0) {
                chunk = std::max<size_t>(1, take / 2);
            } else if (again.empty() && take == chunk) {
                chunk *= 2;
            }
            // the retried pairs first (still largest first), then those not yet run
            again.insert(again.end(), pending.begin() + (std::ptrdiff_t)take, pending.end());
            pending.swap(again);
        }
    }
    al->last_ms = total_ms;
    al->last_launches = launches;
    al->last_cluster_pairs = (int)wide.size();
    al->mem_pair_max = 0, al->mem_total = 0;
    for (int i = 0; i < n; ++i) {
        al->mem_pair_max = std::max<int64_t>(al->mem_pair_max, al->outs[i].mem_bytes);
        al->mem_total += al->outs[i].mem_bytes;
    }
    return AW_OK;
}

static int fetch_ops(wavefront_aligner_gpu *al, int n) {
    int64_t ob = 0;
    for (int i = 0; i < n; ++i) ob = std::max<int64_t>(ob, al->pairs[i].ops_off + al->pairs[i].plen + al->pairs[i].tlen + 8);
    WCUDA(al->h_ops.ensure((size_t)ob + 64));
    WCUDA(cudaMemcpyAsync(al->h_ops.p, al->d_ops.p, (size_t)ob, cudaMemcpyDeviceToHost, al->st));
    WCUDA(cudaStreamSynchronize(al->st));
    return AW_OK;
}

static int public_status(int st) {
    if (st == WFA_RETRY || st == WFA_OVERFLOW) return WFA_OOM;
    return st;
}

extern "C" {

wavefront_aligner_gpu_t *wavefront_aligner_new_gpu(const wavefront_gpu_attr_t *attr) {
    if (!attr) {
        set_error("wavefront_aligner_new_gpu: attributes required");
        return nullptr;
    }
    // wavefront/wavefront_penalties.c:141-150
    if (attr->mismatch <= 0 || attr->gap_opening1 < 0 || attr->gap_extension1 <= 0 || attr->gap_opening2 < 0 ||
        attr->gap_extension2 <= 0) {
        set_error("wavefront_aligner_new_gpu: penalties must be X>0, O1>=0, E1>0, O2>=0, E2>0");
        return nullptr;
    }
    if (attr->memory_mode < 0 || attr->memory_mode > 2) {
        set_error("wavefront_aligner_new_gpu: memory_mode must be 0 (high), 1 (medium) or 2 (low)");
        return nullptr;
    }
    wavefront_aligner_gpu *al = new wavefront_aligner_gpu();
    al->attr = *attr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&al->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaStreamCreateWithFlags(&al->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&al->e0) != cudaSuccess || cudaEventCreate(&al->e1) != cudaSuccess) {
        set_error("wavefront_aligner_new_gpu: CUDA initialisation failed");
        delete al;
        return nullptr;
    }
    return al;
}

void wavefront_aligner_delete_gpu(wavefront_aligner_gpu_t *al) { delete al; }

int wavefront_gpu_last_launches(const wavefront_aligner_gpu_t *al, int *launches, int *cluster_launches,
                                int *cluster_pairs) {
    if (!al) return AW_E_INVAL;
    if (launches) *launches = al->last_launches;
    if (cluster_launches) *cluster_launches = al->last_cluster_launches;
    if (cluster_pairs) *cluster_pairs = al->last_cluster_pairs;
    return AW_OK;
}

void aw_set_wfa_long(int min_length_sum) {
    if (min_length_sum >= 0) g_long_sum.store(min_length_sum);
}

void aw_set_wfa_wide(int width, int tail_width, int cluster_ctas) {
    if (width >= 0) g_wide_width.store(width);
    if (tail_width >= 0) g_wide_tail.store(tail_width);
    if (cluster_ctas > 0) g_wide_cluster.store(std::min(8, cluster_ctas));
}

int wavefront_align_gpu(wavefront_aligner_gpu_t *al, const char *pattern, int pattern_length, const char *text,
                        int text_length) {
    if (!al || pattern_length < 0 || text_length < 0 || (pattern_length > 0 && !pattern) ||
        (text_length > 0 && !text))
        return AW_E_INVAL;
    al->ops.clear();
    al->score = 0;
    const int rc = run_batch(al, 1, &pattern, &pattern_length, &text, &text_length);
    if (rc) return rc;
    const WfaOutDev &o = al->outs[0];
    if (o.status == WFA_COMPLETED) {
        if (fetch_ops(al, 1)) return AW_E_CUDA;
        al->ops.assign((const char *)al->h_ops.p + al->pairs[0].ops_off, (size_t)o.n_ops);
        al->score = o.score;
    }
    return public_status(o.status);
}

int wavefront_gpu_memory(const wavefront_aligner_gpu_t *al, int64_t *pair_max, int64_t *total) {
    if (!al) return AW_E_INVAL;
    if (pair_max) *pair_max = al->mem_pair_max;
    if (total) *total = al->mem_total;
    return AW_OK;
}

int wavefront_gpu_cigar(const wavefront_aligner_gpu_t *al, const char **operations, int *num_operations,
                        int *score) {
    if (!al) return AW_E_INVAL;
    if (operations) *operations = al->ops.c_str();
    if (num_operations) *num_operations = (int)al->ops.size();
    if (score) *score = al->score;
    return AW_OK;
}

int wavefront_align_batch_gpu(wavefront_aligner_gpu_t *al, int n, const char *const *pattern,
                              const int *pattern_length, const char *const *text, const int *text_length,
                              int *status, int *score, int64_t *ops_offset, int *n_ops, char *ops,
                              int64_t ops_capacity, float *device_ms) {
    if (!al || n < 0 || (n > 0 && (!pattern || !pattern_length || !text || !text_length || !status || !score)))
        return AW_E_INVAL;
    if (n == 0) return AW_OK;
    int64_t need = 0;
    for (int i = 0; i < n; ++i) need += (int64_t)pattern_length[i] + text_length[i];
    if (ops && ops_capacity < need) {
        set_error("wavefront_align_batch_gpu: ops buffer needs sum(plen + tlen) bytes");
        return AW_E_INVAL;
    }
    const int rc = run_batch(al, n, pattern, pattern_length, text, text_length);
    if (rc) return rc;
    if (device_ms) *device_ms = al->last_ms;
    if (ops && fetch_ops(al, n)) return AW_E_CUDA;
    int64_t pos = 0;
    for (int i = 0; i < n; ++i) {
        const WfaOutDev &o = al->outs[i];
        status[i] = public_status(o.status);
        score[i] = o.status == WFA_COMPLETED ? o.score : 0;
        const int nops = o.status == WFA_COMPLETED ? o.n_ops : 0;
        if (n_ops) n_ops[i] = nops;
        if (ops_offset) ops_offset[i] = pos;
        if (ops && nops) memcpy(ops + pos, (const char *)al->h_ops.p + al->pairs[i].ops_off, (size_t)nops);
        pos += nops;
    }
    return AW_OK;
}

}  // extern "C"
