// Serving form of the alignment stage: a request loop with continuous batching
// that stands in for AnchorWave's CPU alignment thread pool
// (src/service/AnchorTaskExecutor.h:54-160, ParallelGapBatchScheduler.h:39-280).
//
//   * aw_serve_submit() / aw_serve_submit_route() enqueue one interval as the anchor
//     stage emits it, with the engine the caller's selector chose for it (KSW2
//     full/banded, KSW2 Singletrack, WFA in its four memory modes, score-certified KSW2,
//     sliding-window KSW2) and that engine's parameters;
//   * `slots` worker threads each own their CUDA streams and pooled device
//     buffers (the thread-local pools of the batch entries); requests wait in one
//     FIFO per engine/parameter class, and an idle worker takes the class whose
//     head waited longest, up to max_batch of its requests, as one micro-batch,
//     so requests that arrive while others run on the GPU
//     are admitted as soon as a worker and memory are free, and the micro-batches
//     of different workers overlap on the device;
//   * admission: each request carries its predicted device bytes (traceback or
//     wavefronts); a micro-batch is admitted only while the in-flight total stays
//     under the HBM budget (the -M envelope of AlignmentResourceScheduler.cpp:706
//     restated for device memory); a request that alone exceeds it runs alone;
//   * aw_serve_poll() releases results strictly in request-id order (ids are
//     consecutive from 0, like the gap order of resultBeforeAnchor,
//     ParallelGapBatchScheduler.h:141-209), so the MAF writer sees the same
//     sequence of alignments whatever the batching;
//   * every result is computed by the same kernels as a standalone call, so it is
//     identical alone and in the mix.
#include "aw_internal.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

using namespace aw;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t id;
    int method, band, band_max;
    int64_t window;
    std::string q, t;  // ASCII
    int64_t pred;
    double t_submit;
    int generic;  // KSW2: a base outside ACGT (generic scoring), computed at submit
    int bucket;   // length class: requests of one class share a micro-batch
};

// Length classes keep short intervals out of micro-batches that a long interval
// would hold for the whole of its (much longer) alignment.
int length_bucket(int64_t len) { return len <= 4000 ? 0 : len <= 20000 ? 1 : 2; }

struct Res {
    aw_serve_result_t r;
    double t_done;
};

int64_t predict_bytes(const Req &rq) {
    const int64_t ql = (int64_t)rq.q.size(), tl = (int64_t)rq.t.size();
    if (rq.method == AW_ROUTE_KSW2_CERTIFIED) {
        // the largest banded traceback of the certification (the score pass keeps none)
        const int64_t n = std::min(std::min(ql, tl), (int64_t)std::max(rq.band, rq.band_max) + 1);
        return (ql + tl) * ((n + 63) / 64 + 1) * 64;
    }
    if (rq.method == AW_ROUTE_SLIDING_WINDOW) {
        // one window's full traceback at a time
        const int64_t w = std::max<int64_t>(1, std::min<int64_t>(rq.window + 1, std::max(ql, tl)));
        return ksw_full_tb_bytes((int)std::min<int64_t>(w, ql), (int)std::min<int64_t>(w, tl));
    }
    if (rq.method >= AW_ROUTE_WFA) {
        // wavefront retention grows with the alignment score; a length-based proxy (the
        // piggyback modes keep a ring of recent scores and about 1.6 bytes of blocks per cell)
        const int64_t L = ql + tl;
        return 64 * L + L * L / (rq.method == AW_ROUTE_WFA ? 16 : rq.method == AW_ROUTE_WFA_SINGLETRACK ? 64 : 128);
    }
    if (rq.band >= 0 && rq.band < std::max(ql, tl)) {
        const int64_t n = std::min(std::min(ql, tl), (int64_t)rq.band + 1);
        return (ql + tl) * ((n + 63) / 64 + 1) * 64 * (rq.method == AW_ROUTE_KSW2_SINGLETRACK ? 2 : 1);
    }
    return ksw_full_tb_bytes((int)ql, (int)tl) * (rq.method == AW_ROUTE_KSW2_SINGLETRACK ? 2 : 1);
}

// encodeKswSequence (src/myImportandFunction/alignSlidingWindow.cpp:645-660)
bool encode(const std::string &s, std::vector<uint8_t> &out) {
    bool generic = false;
    out.resize(s.size());
    for (size_t i = 0; i < s.size(); ++i) {
        switch (s[i]) {
        case 'A': case 'a': out[i] = 0; break;
        case 'C': case 'c': out[i] = 1; break;
        case 'G': case 'g': out[i] = 2; break;
        case 'T': case 't': out[i] = 3; break;
        default: out[i] = 4, generic = true; break;
        }
    }
    return generic;
}

}  // namespace

struct aw_server {
    aw_serve_config_t cfg;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    // one FIFO per class (engine, KSW2 scoring flag, length class); popping the front of
    // a class keeps a take O(batch) however long the backlog is
    std::map<std::tuple<int, int, int>, std::deque<Req>> queues;
    size_t queued = 0;
    std::map<uint64_t, Res> done;
    uint64_t next_release = 0;
    int64_t inflight_bytes = 0;
    int busy = 0;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::vector<double> latencies;
    double t_first_submit = -1, t_last_done = 0;
    uint64_t submitted = 0, completed = 0, batches = 0;
    int device = 0;
};

namespace {

// Device memory of one worker: its share of the budget, split between the KSW2 traceback
// arena (50%, reserved when the worker starts) and the wavefront pools of the four WFA
// engines (allocated when an engine first runs; high memory 16%, Singletrack 26% -- the
// engine AnchorWave's selector picks most, for intervals up to tens of kb -- medium and low
// 4% each as they keep a ring and packed-CIGAR blocks), so that the pooled allocations of
// all workers stay inside the budget whatever mix of engines each worker sees.
int64_t worker_share(const aw_server *S) { return S->cfg.hbm_budget / std::max(1, S->cfg.slots); }
int64_t ksw_tb_share(const aw_server *S) { return worker_share(S) * 5 / 10; }
int64_t wfa_pool_share(const aw_server *S, int method) {
    const int pct = method == AW_ROUTE_WFA ? 16 : method == AW_ROUTE_WFA_SINGLETRACK ? 26 : 4;
    return worker_share(S) * pct / 100;
}

// Pops one micro-batch: the requests of the class whose head waited longest, oldest
// first, while they fit the batch size and the budget.
bool take_batch(aw_server *S, std::vector<Req> &batch) {
    batch.clear();
    if (S->queued == 0) return false;
    std::deque<Req> *q = nullptr;
    for (auto &kv : S->queues)
        if (!kv.second.empty() && (!q || kv.second.front().id < q->front().id)) q = &kv.second;
    const int64_t budget = S->cfg.hbm_budget;
    if (S->inflight_bytes > 0 && S->inflight_bytes + q->front().pred > budget) return false;
    // a WFA micro-batch shares one wavefront pool: its predicted bytes stay within that pool,
    // so that large alignments are not started together only to exhaust it and retry
    const int method = q->front().method;
    const int64_t pool = method >= AW_ROUTE_WFA && method <= AW_ROUTE_WFA_LOW ? wfa_pool_share(S, method) : INT64_MAX;
    int64_t bytes = 0;
    while (!q->empty() && (int)batch.size() < S->cfg.max_batch) {
        if (!batch.empty() && S->inflight_bytes + bytes + q->front().pred > budget) break;
        if (!batch.empty() && bytes + q->front().pred > pool) break;
        bytes += q->front().pred;
        batch.push_back(std::move(q->front()));
        q->pop_front();
    }
    S->queued -= batch.size();
    S->inflight_bytes += bytes;
    return true;
}


// Gapped rows -> a KSW2-style CIGAR (M/I/D runs), malloc'd into ez.
void rows_to_cigar(const char *q, const char *d, int64_t n, ksw_extz_t &ez) {
    std::vector<uint32_t> cg;
    int64_t i = 0;
    while (i < n) {
        const uint32_t op = q[i] == '-' ? 2u : d[i] == '-' ? 1u : 0u;
        int64_t j = i + 1;
        while (j < n && (q[j] == '-' ? 2u : d[j] == '-' ? 1u : 0u) == op) ++j;
        cg.push_back((uint32_t)(j - i) << 4 | op);
        i = j;
    }
    ez.n_cigar = ez.m_cigar = (int)cg.size();
    ez.cigar = cg.empty() ? nullptr : (uint32_t *)malloc(sizeof(uint32_t) * cg.size());
    if (ez.cigar) memcpy(ez.cigar, cg.data(), sizeof(uint32_t) * cg.size());
}

// The rescue routes: the batch entries of rescue.cu with the server's scoring in
// AnchorWave's form (mismatch = the matrix's off-diagonal score, gap penalties negative).
void run_rescue_batch(aw_server *S, std::vector<Req> &batch, std::vector<Res> &out) {
    const aw_serve_config_t &C = S->cfg;
    const int n = (int)batch.size();
    const int mis = C.mat[1], o1 = -C.q, e1 = -C.e, o2 = -C.q2, e2 = -C.e2;
    std::vector<const char *> qp(n), dp(n);
    std::vector<int64_t> ql(n), dl(n), b0(n), b1(n), win(n);
    for (int i = 0; i < n; ++i) {
        qp[i] = batch[i].q.data(), dp[i] = batch[i].t.data();
        ql[i] = (int64_t)batch[i].q.size(), dl[i] = (int64_t)batch[i].t.size();
        b0[i] = batch[i].band, b1[i] = batch[i].band_max, win[i] = batch[i].window;
    }
    if (batch[0].method == AW_ROUTE_KSW2_CERTIFIED) {
        std::vector<aw_certified_result_t> r(n);
        const int rc = aw_align_score_certified_batch(n, qp.data(), ql.data(), dp.data(), dl.data(), b0.data(),
                                                      b1.data(), mis, o1, e1, o2, e2, 0.0, nullptr, r.data());
        for (int i = 0; i < n; ++i) {
            out[i].r.status = rc ? rc : r[i].status;
            out[i].r.ez.score = (int)r[i].score;
            if (r[i].alignment_len > 0) rows_to_cigar(r[i].alignment_q, r[i].alignment_d, r[i].alignment_len, out[i].r.ez);
            else if (r[i].best_effort_len > 0)
                rows_to_cigar(r[i].best_effort_q, r[i].best_effort_d, r[i].best_effort_len, out[i].r.ez);
            aw_certified_result_free(&r[i]);
        }
    } else {
        std::vector<aw_window_result_t> r(n);
        const int rc = aw_align_sliding_window_batch(n, qp.data(), ql.data(), dp.data(), dl.data(), win.data(), 0, mis,
                                                     o1, e1, o2, e2, r.data());
        for (int i = 0; i < n; ++i) {
            out[i].r.status = rc;
            out[i].r.ez.score = (int)r[i].score;
            if (r[i].alignment_len > 0) rows_to_cigar(r[i].alignment_q, r[i].alignment_d, r[i].alignment_len, out[i].r.ez);
            aw_window_result_free(&r[i]);
        }
    }
}

void run_batch(aw_server *S, std::vector<Req> &batch, std::vector<Res> &out, wavefront_aligner_gpu_t **al) {
    const aw_serve_config_t &C = S->cfg;
    const int n = (int)batch.size();
    out.assign(n, Res{});
    for (int i = 0; i < n; ++i) {
        memset(&out[i].r, 0, sizeof(aw_serve_result_t));
        out[i].r.id = batch[i].id;
        out[i].r.method = batch[i].method;
    }
    const int method = batch[0].method;
    if (method == AW_ROUTE_KSW2_CERTIFIED || method == AW_ROUTE_SLIDING_WINDOW) {
        run_rescue_batch(S, batch, out);
    } else if (method == AW_ROUTE_KSW2 || method == AW_ROUTE_KSW2_SINGLETRACK) {
        std::vector<std::vector<uint8_t>> qs(n), ts(n);
        bool generic = false;
        for (int i = 0; i < n; ++i) generic |= encode(batch[i].q, qs[i]), generic |= encode(batch[i].t, ts[i]);
        std::vector<const uint8_t *> qp(n), tp(n);
        std::vector<int> ql(n), tl(n), w(n);
        for (int i = 0; i < n; ++i) {
            qp[i] = qs[i].data(), tp[i] = ts[i].data();
            ql[i] = (int)qs[i].size(), tl[i] = (int)ts[i].size(), w[i] = batch[i].band;
        }
        std::vector<ksw_extz_t> ez(n);
        memset(ez.data(), 0, sizeof(ksw_extz_t) * n);
        int flag = generic ? AW_EZ_GENERIC_SC : 0;
        if (method == AW_ROUTE_KSW2_SINGLETRACK) flag |= AW_EZ_SINGLETRACK;
        int rc = aw_ksw_extd2_batch(n, ql.data(), qp.data(), tl.data(), tp.data(), w.data(), C.m, C.mat, C.q, C.e,
                                    C.q2, C.e2, -1, 0, flag, ez.data());
        if (rc == AW_E_CUDA || rc == AW_E_NOMEM) {
            // device memory taken meanwhile (fragmentation, another process): give back the
            // pooled buffers and run the batch once more
            for (int i = 0; i < n; ++i) free(ez[i].cigar);
            memset(ez.data(), 0, sizeof(ksw_extz_t) * n);
            aw_release_thread_buffers();
            rc = aw_ksw_extd2_batch(n, ql.data(), qp.data(), tl.data(), tp.data(), w.data(), C.m, C.mat, C.q, C.e,
                                    C.q2, C.e2, -1, 0, flag, ez.data());
        }
        for (int i = 0; i < n; ++i) {
            out[i].r.status = rc;
            out[i].r.ez = ez[i];
        }
    } else {
        wavefront_gpu_attr_t a;
        a.mismatch = C.wfa_x, a.gap_opening1 = C.wfa_o1, a.gap_extension1 = C.wfa_e1;
        a.gap_opening2 = C.wfa_o2, a.gap_extension2 = C.wfa_e2;
        a.singletrack = method == AW_ROUTE_WFA_SINGLETRACK;
        a.memory_mode = method == AW_ROUTE_WFA_MEDIUM ? 1 : method == AW_ROUTE_WFA_LOW ? 2 : 0;
        // wavefront pool of this engine in this worker: its part of the worker's share
        a.max_memory_abort = std::max<int64_t>(wfa_pool_share(S, method), (int64_t)1 << 26);
        // one aligner per worker and engine, kept for the worker's lifetime
        wavefront_aligner_gpu_t *&A = al[method - AW_ROUTE_WFA];
        if (!A) A = wavefront_aligner_new_gpu(&a);
        std::vector<const char *> pp(n), tp(n);
        std::vector<int> pl(n), tl(n), st(n), sc(n), no(n);
        std::vector<int64_t> off(n);
        int64_t cap = 0;
        for (int i = 0; i < n; ++i) {
            pp[i] = batch[i].t.data(), tp[i] = batch[i].q.data();  // pattern = reference, text = query
            pl[i] = (int)batch[i].t.size(), tl[i] = (int)batch[i].q.size();
            cap += (int64_t)pl[i] + tl[i];
        }
        std::vector<char> ops((size_t)cap + 1);
        const int rc = A ? wavefront_align_batch_gpu(A, n, pp.data(), pl.data(), tp.data(), tl.data(), st.data(),
                                                     sc.data(), off.data(), no.data(), ops.data(), cap + 1, nullptr)
                         : AW_E_CUDA;
        for (int i = 0; i < n; ++i) {
            out[i].r.status = rc ? rc : st[i];
            out[i].r.wfa_score = rc ? 0 : sc[i];
            out[i].r.n_ops = rc ? 0 : no[i];
            if (!rc && no[i] > 0) {
                out[i].r.ops = (char *)malloc((size_t)no[i] + 1);
                memcpy(out[i].r.ops, ops.data() + off[i], (size_t)no[i]);
                out[i].r.ops[no[i]] = 0;
            }
        }
    }
}

void worker_main(aw_server *S, int slot) {
    cudaSetDevice(S->device);
    // each worker's batches get an equal share of the device budget
    const int64_t tb = std::max<int64_t>(ksw_tb_share(S), (int64_t)1 << 26);
    set_thread_tb_budget(tb);
    reserve_thread_tb(tb);
    std::vector<Req> batch;
    std::vector<Res> res;
    wavefront_aligner_gpu_t *al[4] = {nullptr, nullptr, nullptr, nullptr};
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stopping || (S->queued > 0 && take_batch(S, batch)); });
            if (batch.empty() && S->stopping) {
                lk.unlock();
                for (wavefront_aligner_gpu_t *a : al) wavefront_aligner_delete_gpu(a);
                return;
            }
            ++S->busy;
            ++S->batches;
        }
        run_batch(S, batch, res, al);
        const double t = now_s();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            int64_t bytes = 0;
            for (size_t i = 0; i < batch.size(); ++i) {
                bytes += batch[i].pred;
                res[i].r.latency_s = t - batch[i].t_submit;
                res[i].t_done = t;
                S->latencies.push_back(res[i].r.latency_s);
                S->done[batch[i].id] = res[i];
            }
            S->inflight_bytes -= bytes;
            S->completed += batch.size();
            S->t_last_done = t;
            --S->busy;
            batch.clear();
        }
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
    (void)slot;
}

}  // namespace

extern "C" {

aw_server_t *aw_serve_open(const aw_serve_config_t *cfg) {
    if (!cfg || cfg->slots < 1 || cfg->max_batch < 1 || cfg->m < 2 || cfg->m > 8) {
        set_error("aw_serve_open: invalid configuration");
        return nullptr;
    }
    aw_server *S = new aw_server();
    S->cfg = *cfg;
    if (cudaGetDevice(&S->device) != cudaSuccess) {
        set_error("aw_serve_open: no CUDA device");
        delete S;
        return nullptr;
    }
    if (S->cfg.hbm_budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        S->cfg.hbm_budget = (int64_t)(fr * 0.7);
    }
    for (int i = 0; i < cfg->slots; ++i) S->workers.emplace_back(worker_main, S, i);
    return S;
}

int aw_serve_submit(aw_server_t *S, uint64_t id, int method, int band, const char *query, int qlen,
                    const char *target, int tlen) {
    aw_serve_route_t rt;
    rt.method = method, rt.band = band, rt.band_max = -1, rt.window = 0, rt.predicted_bytes = 0;
    return aw_serve_submit_route(S, id, &rt, query, qlen, target, tlen);
}

int aw_serve_submit_route(aw_server_t *S, uint64_t id, const aw_serve_route_t *route, const char *query, int qlen,
                          const char *target, int tlen) {
    if (!S || !route || qlen < 0 || tlen < 0 || route->method < AW_ROUTE_KSW2 ||
        route->method > AW_ROUTE_SLIDING_WINDOW)
        return AW_E_INVAL;
    const int method = route->method;
    if (method == AW_ROUTE_SLIDING_WINDOW && route->window <= 0) {
        set_error("aw_serve_submit_route: the sliding-window route needs window > 0");
        return AW_E_INVAL;
    }
    Req r;
    r.id = id, r.method = method, r.band = route->band, r.band_max = route->band_max, r.window = route->window;
    r.q.assign(query ? query : "", (size_t)qlen);
    r.t.assign(target ? target : "", (size_t)tlen);
    r.pred = predict_bytes(r);
    // the selector's memory estimate of a WFA alignment (its score model) replaces the
    // length-based proxy; KSW2 tracebacks are sized exactly by the server itself
    if (method >= AW_ROUTE_WFA && method <= AW_ROUTE_WFA_LOW && route->predicted_bytes > 0)
        r.pred = route->predicted_bytes;
    r.generic = 0;
    if (method <= AW_ROUTE_KSW2_SINGLETRACK) {
        std::vector<uint8_t> tmp;
        r.generic = (encode(r.q, tmp) | encode(r.t, tmp)) ? 1 : 0;
    }
    r.bucket = length_bucket(std::max<int64_t>(qlen, tlen));
    r.t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->t_first_submit < 0) S->t_first_submit = r.t_submit;
        const auto key = std::make_tuple(r.method, r.generic, r.bucket);
        S->queues[key].push_back(std::move(r));
        ++S->queued;
        ++S->submitted;
    }
    S->cv_work.notify_one();
    return AW_OK;
}

int aw_serve_poll(aw_server_t *S, aw_serve_result_t *out, int max, int wait_ms) {
    if (!S || !out || max < 1) return AW_E_INVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    if (wait_ms > 0)
        S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms),
                            [&] { return S->done.count(S->next_release) > 0; });
    int n = 0;
    while (n < max) {
        auto it = S->done.find(S->next_release);
        if (it == S->done.end()) break;
        out[n++] = it->second.r;
        S->done.erase(it);
        ++S->next_release;
    }
    return n;
}

int aw_serve_stats(aw_server_t *S, aw_serve_stats_t *st) {
    if (!S || !st) return AW_E_INVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->micro_batches = S->batches;
    st->queued = (uint64_t)S->queued;
    st->inflight_bytes = S->inflight_bytes;
    std::vector<double> l = S->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    st->latency_p50_s = pct(0.50);
    st->latency_p99_s = pct(0.99);
    st->elapsed_s = S->t_first_submit < 0 ? 0.0 : S->t_last_done - S->t_first_submit;
    return AW_OK;
}

void aw_serve_close(aw_server_t *S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers) t.join();
    for (auto &kv : S->done) {
        free(kv.second.r.ez.cigar);
        free(kv.second.r.ops);
    }
    delete S;
}

void aw_serve_result_free(aw_serve_result_t *r) {
    if (!r) return;
    free(r->ez.cigar);
    free(r->ops);
    r->ez.cigar = nullptr;
    r->ops = nullptr;
}

}  // extern "C"
