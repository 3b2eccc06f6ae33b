// C-ABI host layer for the KSW2 kernels (drop-in ksw_extd2 entries, batch and
// plan APIs).  Host-side responsibilities:
//   * the argument checks and early returns of ksw_extd2 (minimap2/ksw2_extd2_sse.c:80-105,
//     ksw2_extd2_avx.c:129-133), done before any device work;
//   * routing each pair to the full-matrix strip kernel or to the exact
//     anti-diagonal kernel (banded / Singletrack / z-drop / other flags);
//   * batch planning: pairs sorted largest first, traceback arenas packed into
//     waves under an HBM budget (the -M admission envelope of
//     AlignmentResourceScheduler.cpp:706 restated for device memory);
//   * per-thread pooled device/pinned buffers (grow-only) and a private stream
//     pair, so concurrent host threads never share state (the reference's
//     one-call-per-worker threading contract: each AnchorTaskExecutor worker
//     calls ksw_extd2 on its own, src/service/AnchorTaskExecutor.cpp:54, :374);
//   * CIGAR ownership exactly as ksw_push_cigar (minimap2/ksw2.h:144-154).
#include "aw_internal.h"
#include "ksw2_band.h"
#include "ksw2_exact.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace aw {

// ---- diagnostics -----------------------------------------------------------
static thread_local std::string tls_err;
void set_error(const char *s) {
    tls_err = s;
    if (getenv("AW_VERBOSE")) fprintf(stderr, "[aw_b200] %s\n", s);
}
static void set_error(const std::string &s) { set_error(s.c_str()); }

// ---- cooperative stop ------------------------------------------------------
// The calling thread's deadline, the state ksw_set_progress_callback keeps per thread
// (minimap2/ksw2_progress.c:11-13) when AnchorWave's ScopedKswDeadline installs its
// probe (alignSlidingWindow.cpp:593-640).
static thread_local bool tls_has_deadline = false;
static thread_local std::chrono::steady_clock::time_point tls_deadline;

// Set while this thread captures a plan into a CUDA graph: the timing events then become
// event-record nodes of the graph, so they still time every replay.
static thread_local bool tls_capturing = false;
static cudaError_t record_timing(cudaEvent_t e, cudaStream_t st) {
    return tls_capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
}
#define AW_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            set_error(std::string(#call) + ": " + cudaGetErrorString(_e));              \
            return AW_E_CUDA;                                                           \
        }                                                                               \
    } while (0)

// ---- tuning ----------------------------------------------------------------
static int64_t g_tb_budget = 0;           // 0 = 60% of free memory
static thread_local int64_t tls_tb_budget = 0;  // per-thread override (serving workers)
static thread_local bool tls_all_large = false;  // single-pair calls: every pair gets a warp group
// full-matrix pairs on the critical path go to the banded kernel at full width
// (aw_set_full_pair_routing)
static std::atomic<bool> g_band_full_pairs{true};
static int g_large_warps = 8;
static int g_large_tlen = 4096;
static int g_band_nc = 0;  // banded kernel columns per lane: 0 = chosen per plan, 4 or 8
static std::mutex g_cfg_mu;

// ---- pooled buffers ----------------------------------------------------------
struct PinBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max(n + n / 2, (size_t)4096);
        cudaError_t e = cudaMallocHost(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr, cap = 0;
    }
    template <class T> T *as() const { return (T *)p; }
};

struct Buffers {
    DevBuf qcodes, tcodes, pairs, order, out, cig, packed, packed_off, tb, bnd, queue, error;
    DevBuf exact_ws, deadline;
    DevBuf band_pairs, band_strips, band_units, band_res, band_progress, band_bnd, band_queue, band_walk, band_groups;
    PinBuf h_band;
    PinBuf h_codes, h_pairs, h_order, h_out, h_packed, h_packed_off, h_small;
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    std::vector<cudaEvent_t> ev_k;  // per-launch timing events
    int device = -1;
    int sms = 0;
    ~Buffers() {
        qcodes.release(); tcodes.release(); pairs.release(); order.release(); out.release();
        cig.release(); packed.release(); packed_off.release(); tb.release(); bnd.release();
        queue.release(); error.release(); exact_ws.release(); deadline.release();
        band_pairs.release(); band_strips.release(); band_units.release(); band_res.release();
        band_progress.release(); band_bnd.release(); band_queue.release(); band_walk.release(); h_band.release();
        band_groups.release();
        h_codes.release(); h_pairs.release(); h_order.release(); h_out.release();
        h_packed.release(); h_packed_off.release(); h_small.release();
        for (auto e : ev_k) cudaEventDestroy(e);
        if (ev_a) cudaEventDestroy(ev_a);
        if (ev_b) cudaEventDestroy(ev_b);
        if (ev_t0) cudaEventDestroy(ev_t0);
        if (ev_t1) cudaEventDestroy(ev_t1);
        if (st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
    }
    int init() {
        if (st) return AW_OK;
        AW_CUDA(cudaGetDevice(&device));
        AW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        AW_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        AW_CUDA(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        AW_CUDA(cudaEventCreateWithFlags(&ev_a, cudaEventDisableTiming));
        AW_CUDA(cudaEventCreateWithFlags(&ev_b, cudaEventDisableTiming));
        AW_CUDA(cudaEventCreate(&ev_t0));
        AW_CUDA(cudaEventCreate(&ev_t1));
        return AW_OK;
    }
};

static thread_local Buffers *tls_buf = nullptr;
static Buffers *thread_buffers() {
    if (!tls_buf) {
        tls_buf = new Buffers();
        // released when the thread exits
        static thread_local struct Reaper {
            ~Reaper() { delete tls_buf; tls_buf = nullptr; }
        } reaper;
        (void)reaper;
    }
    return tls_buf;
}

// ---- per-pair routing ----------------------------------------------------------
struct Params {
    int8_t m;
    int8_t mat[64];
    int q, e, q2, e2;   // after the swap
    int zdrop, end_bonus, flag;
    int min_sc, max_sc;
    int qe_pre;         // q+e before the swap
    bool early_return;  // -min_sc > 2(q+e): ksw2_extd2_sse.c:105
};

static bool make_params(int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                        int zdrop, int end_bonus, int flag, Params &P) {
    if (m < 2 || m > 8) return false;
    P.m = m;
    memset(P.mat, 0, sizeof(P.mat));
    memcpy(P.mat, mat, (size_t)m * m);
    int qq = q, ee = e, qq2 = q2, ee2 = e2;
    P.qe_pre = q + e;
    if (qq2 + ee2 < qq + ee) std::swap(qq, qq2), std::swap(ee, ee2);
    P.q = qq, P.e = ee, P.q2 = qq2, P.e2 = ee2;
    P.zdrop = zdrop, P.end_bonus = end_bonus, P.flag = flag;
    P.max_sc = mat[0], P.min_sc = mat[1];
    for (int t = 1; t < m * m; ++t) P.max_sc = std::max<int>(P.max_sc, mat[t]), P.min_sc = std::min<int>(P.min_sc, mat[t]);
    P.early_return = -P.min_sc > 2 * (P.q + P.e);
    return true;
}

static KswScore make_score(const Params &P) {
    KswScore S;
    S.q = P.q, S.e = P.e, S.q2 = P.q2, S.e2 = P.e2;
    S.qe = P.q + P.e, S.qe2 = P.q2 + P.e2;
    S.qe_pre = P.qe_pre;
    S.mch = P.mat[0];
    int lt = P.e != P.e2 ? (P.q2 - P.q) / (P.e - P.e2) - 1 : 0;
    if (P.q2 + P.e2 + lt * P.e2 > P.q + P.e + lt * P.e) ++lt;
    S.long_thres = lt;
    S.long_diff = lt * (P.e - P.e2) - (P.q2 - P.q) - P.e2;
    const int m = P.m;
    const int8_t scN = P.mat[m * m - 1] == 0 ? (int8_t)(-P.e2) : P.mat[m * m - 1];
    for (int tc = 0; tc < 8; ++tc) {
        uint8_t row[8];
        for (int qc = 0; qc < 8; ++qc) {
            int8_t v;
            if (P.flag & AW_EZ_GENERIC_SC)
                v = (tc < m && qc < m) ? P.mat[tc * m + qc] : 0;
            else {
                v = tc == qc ? P.mat[0] : P.mat[1];
                if (tc == m - 1 || qc == m - 1) v = scN;
            }
            row[qc] = (uint8_t)v;
        }
        memcpy(&S.tab_lo[tc], row, 4);
        memcpy(&S.tab_hi[tc], row + 4, 4);
    }
    return S;
}

// The strip kernel computes in 16-bit fields (two cells per register).  It is
// exact when the int8 intermediates of the reference never wrap and when none of
// the features it omits (band, z-drop, max tracking, Singletrack, approximate
// max, extension end) is requested.  The magnitude bound below keeps every
// intermediate of the recurrence (a, b, a2, b2 before and after the z
// adjustment, u, v, x, y, x2, y2) inside int8 for the invariant ranges x,y in
// [-(q+e),-e], x2,y2 in [-(q2+e2),-e2], u,v in [-(q+e), mch+(q+e)], and inside
// the kernel's field biases.
static bool full_path_ok(const Params &P, int qlen, int tlen, int w) {
    if (exact_stop_enabled()) return false;
    const int allowed = AW_EZ_SCORE_ONLY | AW_EZ_RIGHT | AW_EZ_GENERIC_SC | AW_EZ_REV_CIGAR |
                        AW_EZ_SEMIGLOBAL_END;
    if (P.flag & ~allowed) return false;
    if (!(w < 0 || w >= std::max(qlen, tlen))) return false;
    if (P.zdrop >= 0) return false;
    if (P.max_sc > 0 || P.mat[0] < P.max_sc) return false;
    if (P.q < 0 || P.e < 0 || P.q2 < 0 || P.e2 < 0) return false;
    if (P.e2 > P.e || P.q2 < P.q) return false;
    const int mag = (P.q2 + P.e2) + (P.q + P.e) + std::abs(P.min_sc) + std::abs((int)P.mat[0]);
    if (mag > 100) return false;
    const int64_t nstrip = (tlen + KSW_STRIP - 1) / KSW_STRIP;
    if (nstrip * ((int64_t)qlen + 2) + qlen > INT_MAX / 2) return false;
    return true;
}

// The banded strip kernel (ksw2_band.cu) restates the reference's padding-lane
// semantics, so it takes any band and the Singletrack traceback (both entries: the AVX
// one and ksw_extd2_singletrack_sse with its 16-byte blocks and end rules); it shares
// the strip kernel's scoring restrictions (no z-drop or max tracking: with mat <= 0
// every H is <= 0, so ez->max stays 0 and max_t/max_q stay -1).
static bool band_path_ok(const Params &P, int qlen, int tlen) {
    if (exact_stop_enabled()) return false;
    const int allowed = AW_EZ_SCORE_ONLY | AW_EZ_RIGHT | AW_EZ_GENERIC_SC | AW_EZ_REV_CIGAR |
                        AW_EZ_SEMIGLOBAL_END | AW_EZ_SINGLETRACK | AW_EZ_SSE_SINGLETRACK;
    if (P.flag & ~allowed) return false;
    if (P.zdrop >= 0) return false;
    if (P.max_sc > 0 || P.mat[0] < P.max_sc) return false;
    if (P.q < 0 || P.e < 0 || P.q2 < 0 || P.e2 < 0) return false;
    if (P.e2 > P.e || P.q2 < P.q) return false;
    const int mag = (P.q2 + P.e2) + (P.q + P.e) + std::abs(P.min_sc) + std::abs((int)P.mat[0]);
    if (mag > 100) return false;
    if ((int64_t)qlen + tlen > INT_MAX / 4) return false;
    return true;
}

static void reset_extz(ksw_extz_t *ez) {  // minimap2/ksw2.h:194-199
    ez->max_q = ez->max_t = ez->mqe_t = ez->mte_q = -1;
    ez->max = 0, ez->score = ez->mqe = ez->mte = AW_NEG_INF;
    ez->n_cigar = 0, ez->zdropped = 0, ez->reach_end = 0, ez->stopped = 0;
}

// ---- CIGAR ownership ------------------------------------------------------------
typedef void *(*krealloc_fn)(void *, void *, size_t);
static krealloc_fn find_krealloc() {
    static krealloc_fn fn = (krealloc_fn)dlsym(RTLD_DEFAULT, "krealloc");
    return fn;
}

// Store n words into ez->cigar with the capacity growth ksw_push_cigar would have
// produced (m_cigar doubles from its entry value, starting at 4).
static bool store_cigar(void *km, ksw_extz_t *ez, const uint32_t *words, int n) {
    ez->n_cigar = n;
    if (n == 0) return true;
    int m = ez->m_cigar;
    if (n > m) {
        int mm = m;
        while (mm < n) mm = mm ? mm << 1 : 4;
        void *p;
        if (km) {
            krealloc_fn kr = find_krealloc();
            if (!kr) {
                set_error("km != NULL but no krealloc symbol in the process");
                ez->n_cigar = 0;
                return false;
            }
            p = kr(km, ez->cigar, (size_t)mm << 2);
        } else {
            p = realloc(ez->cigar, (size_t)mm << 2);
        }
        if (!p) {
            ez->n_cigar = 0;
            return false;
        }
        ez->cigar = (uint32_t *)p;
        ez->m_cigar = mm;
    }
    memcpy(ez->cigar, words, (size_t)n * 4);
    return true;
}

}  // namespace aw

using namespace aw;

// ---- plan ----------------------------------------------------------------------------
struct aw_ksw_plan {
    Buffers own;              // used when the plan owns its buffers
    Buffers *B = nullptr;     // buffers in use (own or the thread's pool)
    Params P;
    KswScore S;
    int n = 0;
    std::vector<int> qlen, tlen, w;
    std::vector<int> route;   // 0 = no device work (early return), 1 = strip kernel, 2 = exact kernel, 3 = banded kernel
    std::vector<int> early_zdrop;
    std::vector<KswPair> pairs;
    std::vector<int64_t> qoff, toff;
    int64_t qbytes = 0, tbytes = 0, cig_words = 0;
    // waves of strip-kernel pairs: order array segments
    struct Wave {
        int begin_small, n_small, begin_large, n_large;  // ranges in order[]
        int64_t tb_bytes, bnd_words;
    };
    std::vector<Wave> waves;
    std::vector<int32_t> order;      // strip-kernel processing order, wave by wave
    std::vector<int32_t> exact_ids;  // pairs for the exact kernel
    std::vector<int32_t> band_ids;   // pairs for the banded kernel
    BandPlan band;
    int refused = 0;                 // banded pairs refused for the budget (reported zdropped)
    int64_t tb_cap = 0, bnd_cap = 0;
    int64_t cells = 0, tb_total = 0;
    int launches = 0;
    bool uploaded = false, executed = false;
    float dp_ms = 0.f, bt_ms = 0.f;
    // re-execution through a CUDA graph (aw_ksw_plan_execute): the first execute runs
    // eagerly (lazy set-up of the kernels), the second captures the launch sequence, later
    // ones replay it
    int eager_runs = 0;
    bool graph_off = false, graph_used = false;
    int graph_warps = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr, graph = nullptr;
    }
    ~aw_ksw_plan() { drop_graph(); }
};

// Columns per lane of the banded kernel for this plan: 4 halves the pipeline lag between
// strips (the band edge sweeps a strip in 32*nc rows) at a few percent more work per
// cell; it pays when the plan is bound by the longest pair's chain of strips rather than
// by total work.  Estimates: ~1 us per strip row-step on the chain, ~300 GCUPS of work.
static int band_columns(const aw_ksw_plan_t *pl) {
    int fixed;
    {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        fixed = g_band_nc;
    }
    if (fixed == 4 || fixed == 8) return fixed;
    double work = 0.0, chain = 0.0;
    for (int32_t i : pl->band_ids) {
        const int ql = pl->qlen[i], tl = pl->tlen[i];
        const int ww = pl->w[i] < 0 ? std::max(ql, tl) : std::min(pl->w[i], std::max(ql, tl));
        work += 2.0 * std::min<double>(ww, std::max(ql, tl)) * (double)std::max(ql, tl) / 3e11;
        chain = std::max(chain, (1.25 * tl + 2.0 * ww + 300.0) * 1e-6);
    }
    return chain > work ? 4 : 8;
}

static int plan_build(aw_ksw_plan_t *pl, int n, const int *qlen, const int *tlen, const int *w) {
    pl->n = n;
    pl->qlen.assign(qlen, qlen + n);
    pl->tlen.assign(tlen, tlen + n);
    pl->w.assign(n, -1);
    if (w) pl->w.assign(w, w + n);
    pl->route.assign(n, 0);
    pl->early_zdrop.assign(n, 0);
    pl->pairs.resize(n);
    pl->qoff.resize(n);
    pl->toff.resize(n);
    const Params &P = pl->P;
    int64_t qb = 0, tbt = 0, cw = 0;
    for (int i = 0; i < n; ++i) {
        const int ql = pl->qlen[i], tl = pl->tlen[i];
        pl->qoff[i] = qb, pl->toff[i] = tbt;
        if (ql > 0) qb += ql;
        if (tl > 0) tbt += tl;
        // ksw2_extd2_sse.c:81 / ksw2_extd2_avx.c:129-133 / :105
        if (P.m <= 1 || ql <= 0 || tl <= 0) continue;
        if (ql > INT_MAX - tl + 1) { pl->early_zdrop[i] = 1; continue; }
        if (P.early_return) continue;
        pl->route[i] = full_path_ok(P, ql, tl, pl->w[i]) ? 1 : band_path_ok(P, ql, tl) ? 3 : 2;
        KswPair &kp = pl->pairs[i];
        kp.qoff = pl->qoff[i], kp.toff = pl->toff[i];
        kp.qlen = ql, kp.tlen = tl;
        kp.cig_off = cw;
        kp.tb_off = 0, kp.bnd_off = 0;
        cw += (int64_t)ql + tl + 2;
        pl->cells += (int64_t)ql * tl;
    }
    pl->qbytes = qb, pl->tbytes = tbt, pl->cig_words = cw;
    // A full-matrix pair that would be the batch's critical path goes to the banded strip
    // kernel at full width instead (w >= max(qlen, tlen) is the reference's full mode, so the
    // results are the same): the strip kernel pipelines one pair's strips over a group of
    // 8 warps of one CTA, ceil(strips / 8) sweeps of its rows, while the banded kernel
    // pipelines them across CTAs, one strip per warp.  Estimates (seconds): strip-kernel
    // chain ceil(ceil(tlen/512)/8) * (qlen + 600) * 0.35e-6 against the batch's work at
    // 1e12 cells/s, and the banded kernel's chain (tlen/256 strips * 64 lane-steps * 2e-6, plus
    // the rows) and the pair's work at 2e11 cells/s.
    if (g_band_full_pairs.load()) {
        double work = 0.0;
        for (int i = 0; i < n; ++i)
            if (pl->route[i] == 1) work += (double)pl->qlen[i] * pl->tlen[i];
        const double batch_s = work / 1e12;
        for (int i = 0; i < n; ++i) {
            if (pl->route[i] != 1 || !band_path_ok(P, pl->qlen[i], pl->tlen[i])) continue;
            const double ql = pl->qlen[i], tl = pl->tlen[i];
            const double k1 = std::ceil(std::ceil(tl / KSW_STRIP) / 8.0) * (ql + 600.0) * 0.35e-6;
            const double k2 = std::ceil(tl / 256.0) * 64.0 * 2e-6 + ql * 0.3e-6 + ql * tl / 2e11;
            if (k1 > 1.5 * std::max(batch_s, k2)) pl->route[i] = 3;
        }
    }
    // strip-kernel pairs: largest first, packed into traceback waves
    std::vector<int32_t> strip;
    for (int i = 0; i < n; ++i)
        if (pl->route[i] == 1) strip.push_back(i);
        else if (pl->route[i] == 2) pl->exact_ids.push_back(i);
        else if (pl->route[i] == 3) pl->band_ids.push_back(i);
    std::sort(strip.begin(), strip.end(), [&](int a, int b) {
        const int64_t ca = (int64_t)pl->qlen[a] * pl->tlen[a], cb = (int64_t)pl->qlen[b] * pl->tlen[b];
        return ca != cb ? ca > cb : a < b;
    });
    const bool cigar = !(P.flag & AW_EZ_SCORE_ONLY);
    int64_t budget = tls_tb_budget;
    if (budget <= 0) {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        budget = g_tb_budget;
    }
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = (size_t)16 << 30;
        // the traceback arena this thread already holds is reused (or freed) by this
        // batch, so it counts as available: otherwise every call after the first would
        // see the pooled arena as used memory and split the batch into more waves
        if (pl->B) fr += pl->B->tb.cap;
        budget = (int64_t)(fr * 0.6);
    }
    // LPT multiway partition of traceback bytes into the fewest waves that fit
    std::vector<std::vector<int32_t>> wv;
    std::vector<int64_t> wload, wbnd;
    for (int32_t i : strip) {
        const int64_t tbb = cigar ? ksw_full_tb_bytes(pl->qlen[i], pl->tlen[i]) : 0;
        const int64_t bw = ksw_full_bnd_words(pl->qlen[i], pl->tlen[i]);
        pl->tb_total += tbb;
        if (tbb > budget) {
            set_error("pair traceback exceeds the HBM traceback budget");
            return AW_E_NOMEM;
        }
        int best = -1;
        for (size_t k = 0; k < wv.size(); ++k)
            if (wload[k] + tbb <= budget && (best < 0 || wload[k] < wload[best])) best = (int)k;
        if (best < 0) {
            wv.emplace_back();
            wload.push_back(0);
            wbnd.push_back(0);
            best = (int)wv.size() - 1;
        }
        KswPair &kp = pl->pairs[i];
        kp.tb_off = wload[best];
        kp.bnd_off = wbnd[best];
        wload[best] += (tbb + 255) / 256 * 256;
        wbnd[best] += (bw + 63) / 64 * 64;
        wv[best].push_back(i);
    }
    int large_tlen, large_warps;
    {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        large_tlen = g_large_tlen, large_warps = g_large_warps;
    }
    for (size_t k = 0; k < wv.size(); ++k) {
        aw_ksw_plan::Wave W;
        std::vector<int32_t> lg, sm;
        for (int32_t i : wv[k])
            ((pl->tlen[i] >= large_tlen || tls_all_large) && large_warps > 1 ? lg : sm).push_back(i);
        W.begin_large = (int)pl->order.size();
        W.n_large = (int)lg.size();
        pl->order.insert(pl->order.end(), lg.begin(), lg.end());
        W.begin_small = (int)pl->order.size();
        W.n_small = (int)sm.size();
        pl->order.insert(pl->order.end(), sm.begin(), sm.end());
        W.tb_bytes = wload[k];
        W.bnd_words = wbnd[k];
        pl->tb_cap = std::max(pl->tb_cap, W.tb_bytes);
        pl->bnd_cap = std::max(pl->bnd_cap, W.bnd_words);
        pl->waves.push_back(W);
    }
    if (!pl->band_ids.empty()) {
        std::vector<int32_t> refused;
        // ksw_extd2_singletrack_sse works on 16-byte blocks whatever the build's width
        const bool sse_st = (P.flag & AW_EZ_SINGLETRACK) && (P.flag & AW_EZ_SSE_SINGLETRACK);
        if (band_plan_build(pl->band, pl->band_ids, pl->qlen, pl->tlen, pl->w, pl->pairs, P.flag,
                            sse_st ? 16 : exact_block(), budget, band_columns(pl), &refused)) {
            set_error("pair traceback exceeds the HBM traceback budget");
            return AW_E_NOMEM;
        }
        if (!refused.empty()) {
            // pairs that cannot run within the budget: the reference's allocation-failure
            // result (ksw2_extd2_avx.c:206-210), the other pairs of the batch run as planned
            for (int32_t i : refused) pl->route[i] = 0, pl->early_zdrop[i] = 1;
            pl->band_ids.erase(std::remove_if(pl->band_ids.begin(), pl->band_ids.end(),
                                              [&](int32_t i) { return pl->route[i] != 3; }),
                               pl->band_ids.end());
            pl->refused = (int)refused.size();
            set_error("a pair's traceback does not fit the HBM traceback budget (a Singletrack traceback, which "
                      "cannot be recomputed in strip groups, or a single strip beyond it): pair reported as "
                      "zdropped (allocation failure)");
        }
        pl->tb_cap = std::max(pl->tb_cap, pl->band.tb_cap);
        pl->tb_total += pl->band.tb_total;
    }
    pl->S = make_score(P);
    return AW_OK;
}

static int plan_alloc(aw_ksw_plan_t *pl) {
    Buffers *B = pl->B;
    int rc = B->init();
    if (rc) return rc;
    const int n = pl->n;
    AW_CUDA(B->qcodes.ensure(pl->qbytes + 16));
    AW_CUDA(B->tcodes.ensure(pl->tbytes + 16));
    AW_CUDA(B->pairs.ensure(sizeof(KswPair) * (size_t)std::max(n, 1)));
    AW_CUDA(B->order.ensure(sizeof(int32_t) * (pl->order.size() + pl->exact_ids.size() + 1)));
    AW_CUDA(B->out.ensure(sizeof(KswOut) * (size_t)std::max(n, 1)));
    AW_CUDA(B->cig.ensure(4 * (size_t)(pl->cig_words + 1)));
    AW_CUDA(B->packed.ensure(4 * (size_t)(pl->cig_words + 1)));
    AW_CUDA(B->packed_off.ensure(8 * (size_t)std::max(n, 1)));
    AW_CUDA(B->tb.ensure((size_t)pl->tb_cap + 256));
    AW_CUDA(B->bnd.ensure(4 * (size_t)pl->bnd_cap + 256));
    AW_CUDA(B->queue.ensure(sizeof(int32_t) * 64 * (2 * pl->waves.size() + 2)));  // two counters per wave
    AW_CUDA(B->error.ensure(sizeof(int32_t) * 4));
    if (!pl->band_ids.empty()) {
        const BandPlan &bp = pl->band;
        AW_CUDA(B->band_pairs.ensure(sizeof(BandPairDev) * bp.pairs.size()));
        AW_CUDA(B->band_strips.ensure(sizeof(BandStripDev) * bp.strips.size()));
        AW_CUDA(B->band_units.ensure(sizeof(int2) * bp.units.size()));
        AW_CUDA(B->band_res.ensure(sizeof(BandRes) * bp.pairs.size()));
        AW_CUDA(B->band_walk.ensure(sizeof(BandWalkState) * bp.pairs.size()));
        AW_CUDA(B->band_progress.ensure(sizeof(int32_t) * PROG_STRIDE * bp.strips.size()));
        AW_CUDA(B->band_bnd.ensure(sizeof(uint2) * (size_t)bp.bnd_cap + 256));
        AW_CUDA(B->band_queue.ensure(sizeof(int32_t) * 64 * bp.waves.size()));
        AW_CUDA(B->band_groups.ensure(sizeof(BandGroupDev) * std::max<size_t>(bp.groups.size(), 1)));
    }
    AW_CUDA(B->h_pairs.ensure(sizeof(KswPair) * (size_t)std::max(n, 1)));
    AW_CUDA(B->h_order.ensure(sizeof(int32_t) * (pl->order.size() + pl->exact_ids.size() + 1)));
    AW_CUDA(B->h_out.ensure(sizeof(KswOut) * (size_t)std::max(n, 1)));
    AW_CUDA(B->h_packed_off.ensure(8 * (size_t)std::max(n, 1)));
    return AW_OK;
}

static int plan_upload(aw_ksw_plan_t *pl, const uint8_t *const *query, const uint8_t *const *target) {
    Buffers *B = pl->B;
    const int n = pl->n;
    AW_CUDA(B->h_codes.ensure((size_t)(pl->qbytes + pl->tbytes) + 32));
    uint8_t *hq = B->h_codes.as<uint8_t>(), *ht = hq + pl->qbytes + 16;
    auto stage = [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            if (pl->qlen[i] > 0) memcpy(hq + pl->qoff[i], query[i], (size_t)pl->qlen[i]);
            if (pl->tlen[i] > 0) memcpy(ht + pl->toff[i], target[i], (size_t)pl->tlen[i]);
        }
    };
    // large batches: the staging copy (pageable -> pinned) is split over a few host threads
    const int64_t bytes = pl->qbytes + pl->tbytes;
    const int nt = bytes < ((int64_t)8 << 20) ? 1
                   : (int)std::min<int64_t>({8, (int64_t)std::max(1u, std::thread::hardware_concurrency()), bytes >> 22});
    if (nt <= 1) {
        stage(0, n);
    } else {
        // pairs split by bytes, so every thread copies about the same amount
        std::vector<int> cut(nt + 1, n);
        cut[0] = 0;
        int64_t acc = 0;
        int t = 1;
        for (int i = 0; i < n && t < nt; ++i) {
            acc += std::max(pl->qlen[i], 0) + std::max(pl->tlen[i], 0);
            if (acc >= bytes * t / nt) cut[t++] = i + 1;
        }
        std::vector<std::thread> th;
        for (int k = 1; k < nt; ++k) th.emplace_back(stage, cut[k], cut[k + 1]);
        stage(cut[0], cut[1]);
        for (auto &x : th) x.join();
    }
    memcpy(B->h_pairs.p, pl->pairs.data(), sizeof(KswPair) * (size_t)n);
    int32_t *ho = B->h_order.as<int32_t>();
    std::copy(pl->order.begin(), pl->order.end(), ho);
    std::copy(pl->exact_ids.begin(), pl->exact_ids.end(), ho + pl->order.size());
    AW_CUDA(cudaMemcpyAsync(B->qcodes.p, hq, (size_t)pl->qbytes, cudaMemcpyHostToDevice, B->st));
    AW_CUDA(cudaMemcpyAsync(B->tcodes.p, ht, (size_t)pl->tbytes, cudaMemcpyHostToDevice, B->st));
    AW_CUDA(cudaMemcpyAsync(B->pairs.p, B->h_pairs.p, sizeof(KswPair) * (size_t)n, cudaMemcpyHostToDevice, B->st));
    AW_CUDA(cudaMemcpyAsync(B->order.p, ho, sizeof(int32_t) * (pl->order.size() + pl->exact_ids.size()),
                            cudaMemcpyHostToDevice, B->st));
    if (!pl->band_ids.empty()) {
        const BandPlan &bp = pl->band;
        const size_t np = sizeof(BandPairDev) * bp.pairs.size(), ns = sizeof(BandStripDev) * bp.strips.size(),
                     nu = sizeof(int2) * bp.units.size(), ng = sizeof(BandGroupDev) * bp.groups.size();
        AW_CUDA(B->h_band.ensure(np + ns + nu + ng));
        uint8_t *h = B->h_band.as<uint8_t>();
        memcpy(h, bp.pairs.data(), np);
        memcpy(h + np, bp.strips.data(), ns);
        memcpy(h + np + ns, bp.units.data(), nu);
        if (ng) memcpy(h + np + ns + nu, bp.groups.data(), ng);
        AW_CUDA(cudaMemcpyAsync(B->band_pairs.p, h, np, cudaMemcpyHostToDevice, B->st));
        AW_CUDA(cudaMemcpyAsync(B->band_strips.p, h + np, ns, cudaMemcpyHostToDevice, B->st));
        AW_CUDA(cudaMemcpyAsync(B->band_units.p, h + np + ns, nu, cudaMemcpyHostToDevice, B->st));
        if (ng) AW_CUDA(cudaMemcpyAsync(B->band_groups.p, h + np + ns + nu, ng, cudaMemcpyHostToDevice, B->st));
    }
    pl->uploaded = true;
    return AW_OK;
}

// Enqueues every wave of the plan on its stream (no host synchronisation).
static int plan_launch(aw_ksw_plan_t *pl) {
    Buffers *B = pl->B;
    const Params &P = pl->P;
    if (!pl->uploaded) { set_error("plan not uploaded"); return AW_E_INVAL; }
    const size_t nq = 64 * (2 * pl->waves.size() + 2);  // large + small counter per wave, 256 B apart
    int launches = 0;
    AW_CUDA(cudaMemsetAsync(B->queue.p, 0, sizeof(int32_t) * nq, B->st));
    AW_CUDA(cudaMemsetAsync(B->error.p, 0, sizeof(int32_t) * 4, B->st));
    AW_CUDA(cudaMemsetAsync(B->out.p, 0, sizeof(KswOut) * (size_t)std::max(pl->n, 1), B->st));
    AW_CUDA(record_timing(B->ev_t0, B->st));
    // the deadline word: globaltimer at the start of this work + the time left
    const unsigned long long *deadline = nullptr;
    if (tls_has_deadline) {
        const long long left = std::chrono::duration_cast<std::chrono::nanoseconds>(
                                   tls_deadline - std::chrono::steady_clock::now()).count();
        AW_CUDA(B->deadline.ensure(sizeof(unsigned long long)));
        AW_CUDA(launch_set_deadline(B->deadline.as<unsigned long long>(),
                                    (unsigned long long)std::max(left, 0LL), B->st));
        deadline = B->deadline.as<unsigned long long>();
        ++launches;
    }
    int large_warps;
    {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        large_warps = g_large_warps;
    }
    // per-wave timing events: DP phase start, DP phase end (after the join), backtrack end
    const size_t need_ev = 3 * (pl->waves.size() + pl->band.waves.size()) + 3;
    while (B->ev_k.size() < need_ev) {
        cudaEvent_t e;
        AW_CUDA(cudaEventCreate(&e));
        B->ev_k.push_back(e);
    }
    const int nw = (int)pl->waves.size();
    for (int k = 0; k < nw; ++k) {
        const auto &W = pl->waves[k];
        KswFullArgs a;
        a.qcodes = B->qcodes.as<uint8_t>(), a.tcodes = B->tcodes.as<uint8_t>();
        a.pairs = B->pairs.as<KswPair>(), a.out = B->out.as<KswOut>();
        a.tb = B->tb.as<uint8_t>(), a.bnd = B->bnd.as<uint32_t>();
        a.error = B->error.as<int32_t>();
        a.sc = pl->S;
        a.deadline = deadline;
        AW_CUDA(record_timing(B->ev_k[3 * k], B->st));
        // fork: large pairs on st2 (groups of large_warps warps), small on st (single warps)
        AW_CUDA(cudaEventRecord(B->ev_a, B->st));
        AW_CUDA(cudaStreamWaitEvent(B->st2, B->ev_a, 0));
        if (W.n_large > 0) {
            a.order = B->order.as<int32_t>() + W.begin_large;
            a.n = W.n_large;
            a.queue = B->queue.as<int32_t>() + 64 * (2 * k);
            const int groups = 8 / large_warps;
            const int occ = std::max(1, ksw_full_occupancy(P.flag, large_warps, groups));
            const int ctas = std::min(W.n_large / groups + 1, occ * B->sms);
            AW_CUDA(launch_ksw_full(a, P.flag, large_warps, groups, ctas, B->st2));
            ++launches;
        }
        if (W.n_small > 0) {
            a.order = B->order.as<int32_t>() + W.begin_small;
            a.n = W.n_small;
            a.queue = B->queue.as<int32_t>() + 64 * (2 * k + 1);
            // warps per small pair: one when the pairs alone fill the resident warps, else
            // up to 8 so that a small batch still runs on the whole GPU (a pair's strips
            // then pipeline over its warps instead of running one after another)
            const int resident = 16 * B->sms;  // 2 CTAs x 8 warps per SM
            const int64_t used = std::min<int64_t>((int64_t)W.n_large * large_warps, resident);
            int ws = 1;
            while (ws < 8 && (int64_t)W.n_small * (2 * ws) <= resident - used) ws *= 2;
            const int groups = 8 / ws;
            const int occ = std::max(1, ksw_full_occupancy(P.flag, ws, groups));
            const int ctas = std::min((W.n_small + groups - 1) / groups, occ * B->sms);
            AW_CUDA(launch_ksw_full(a, P.flag, ws, groups, ctas, B->st));
            ++launches;
        }
        AW_CUDA(cudaEventRecord(B->ev_b, B->st2));
        AW_CUDA(cudaStreamWaitEvent(B->st, B->ev_b, 0));
        AW_CUDA(record_timing(B->ev_k[3 * k + 1], B->st));
        if (!(P.flag & AW_EZ_SCORE_ONLY) && W.n_large + W.n_small > 0) {
            AW_CUDA(launch_ksw_backtrack_full(B->pairs.as<KswPair>(), B->order.as<int32_t>() + W.begin_large,
                                              W.n_large + W.n_small, B->tb.as<uint8_t>(), B->out.as<KswOut>(),
                                              B->cig.as<uint32_t>(), P.flag, B->st));
            ++launches;
        }
        AW_CUDA(record_timing(B->ev_k[3 * k + 2], B->st));
    }
    const int nbw = pl->band_ids.empty() ? 0 : (int)pl->band.waves.size();
    if (nbw > 0) {
        BandDev D;
        D.pairs = B->band_pairs.as<BandPairDev>(), D.strips = B->band_strips.as<BandStripDev>();
        D.units = B->band_units.as<int2>(), D.res = B->band_res.as<BandRes>();
        D.walk = B->band_walk.as<BandWalkState>();
        D.progress = B->band_progress.as<int32_t>(), D.queue = B->band_queue.as<int32_t>();
        D.bnd = B->band_bnd.as<uint2>(), D.tb = B->tb.as<uint8_t>(), D.error = B->error.as<int32_t>();
        D.groups = B->band_groups.as<BandGroupDev>();
        D.deadline = deadline;
        const int ctas = band_occupancy(P.flag) * B->sms;
        for (int k = 0; k < nbw; ++k) {
            cudaEvent_t *ev = &B->ev_k[3 * (nw + k)];
            AW_CUDA(record_timing(ev[0], B->st));
            AW_CUDA(band_launch_dp(pl->band, k, D, B->qcodes.as<uint8_t>(), B->tcodes.as<uint8_t>(), pl->S, P.flag,
                                   ctas, B->st));
            AW_CUDA(record_timing(ev[1], B->st));
            AW_CUDA(band_launch_finish(pl->band, k, D, B->qcodes.as<uint8_t>(), B->tcodes.as<uint8_t>(), pl->S,
                                       P.flag, B->out.as<KswOut>(), B->cig.as<uint32_t>(), P.mat, P.m, B->st));
            launches += 2;
            const BandWave &BW = pl->band.waves[k];
            if (BW.nround > 0) {
                AW_CUDA(band_launch_groups(pl->band, k, D, B->qcodes.as<uint8_t>(), B->tcodes.as<uint8_t>(), pl->S,
                                           P.flag, B->out.as<KswOut>(), B->cig.as<uint32_t>(), P.mat, P.m, ctas,
                                           B->st));
                launches += 3 * BW.nround;  // counters, strips, walks per round
            }
            AW_CUDA(record_timing(ev[2], B->st));
        }
    }
    if (!pl->exact_ids.empty()) {
        int rc = run_exact_ksw(pl->exact_ids.size(), B->order.as<int32_t>() + pl->order.size(),
                               B->qcodes.as<uint8_t>(), B->tcodes.as<uint8_t>(), B->pairs.as<KswPair>(),
                               pl->pairs, pl->exact_ids, pl->w, P.m, P.mat, pl->S, P.zdrop, P.end_bonus,
                               P.flag, B->out.as<KswOut>(), B->cig.as<uint32_t>(), B->exact_ws,
                               B->st, &launches, deadline);
        if (rc) return rc;
    }
    AW_CUDA(record_timing(B->ev_t1, B->st));
    pl->launches = launches;
    return AW_OK;
}

// Waits for plan_launch's work, checks the device error flag, collects timings.
static int plan_finish(aw_ksw_plan_t *pl, float *ms) {
    Buffers *B = pl->B;
    const int nw = (int)(pl->waves.size() + (pl->band_ids.empty() ? 0 : pl->band.waves.size()));
    AW_CUDA(cudaStreamSynchronize(B->st));
    int32_t err = 0;
    AW_CUDA(cudaMemcpy(&err, B->error.p, 4, cudaMemcpyDeviceToHost));
    if (err) { set_error("a bounded device wait gave up (pipeline stall)"); return AW_E_TIMEOUT; }
    if (ms) AW_CUDA(cudaEventElapsedTime(ms, B->ev_t0, B->ev_t1));
    float dp = 0.f, bt = 0.f;
    for (int k = 0; k < nw; ++k) {
        float t0 = 0.f, t1 = 0.f;
        AW_CUDA(cudaEventElapsedTime(&t0, B->ev_k[3 * k], B->ev_k[3 * k + 1]));
        AW_CUDA(cudaEventElapsedTime(&t1, B->ev_k[3 * k + 1], B->ev_k[3 * k + 2]));
        dp += t0, bt += t1;
        const int kb = k - (int)pl->waves.size();
        if (kb >= 0 && getenv("AW_VERBOSE")) {
            const BandWave &BW = pl->band.waves[kb];
            fprintf(stderr, "[aw_b200] band wave %d: %d pairs, %d units, traceback %.1f GB, %d recompute rounds; "
                            "DP %.1f ms, traceback and rounds %.1f ms\n",
                    kb, BW.npair, BW.nunit, BW.tb_bytes / 1e9, BW.nround, t0, t1);
        }
    }
    pl->dp_ms = dp;
    pl->bt_ms = bt;
    pl->executed = true;
    return AW_OK;
}

static int plan_execute(aw_ksw_plan_t *pl, float *ms) {
    const int rc = plan_launch(pl);
    return rc ? rc : plan_finish(pl, ms);
}

static int plan_download(aw_ksw_plan_t *pl, ksw_extz_t *ez, void *km) {
    Buffers *B = pl->B;
    const int n = pl->n;
    if (!pl->executed) { set_error("plan not executed"); return AW_E_INVAL; }
    AW_CUDA(cudaMemcpyAsync(B->h_out.p, B->out.p, sizeof(KswOut) * (size_t)n, cudaMemcpyDeviceToHost, B->st));
    AW_CUDA(cudaStreamSynchronize(B->st));
    const KswOut *ho = B->h_out.as<KswOut>();
    const bool cigar = !(pl->P.flag & AW_EZ_SCORE_ONLY);
    int64_t total = 0;
    int64_t *poff = B->h_packed_off.as<int64_t>();
    for (int i = 0; i < n; ++i) {
        poff[i] = total;
        if (pl->route[i] && cigar) total += ho[i].n_cigar;
    }
    if (cigar && total > 0) {
        AW_CUDA(cudaMemcpyAsync(B->packed_off.p, poff, 8 * (size_t)n, cudaMemcpyHostToDevice, B->st));
        AW_CUDA(launch_ksw_pack_cigar(B->pairs.as<KswPair>(), n, B->out.as<KswOut>(), B->cig.as<uint32_t>(),
                                      B->packed_off.as<int64_t>(), B->packed.as<uint32_t>(), B->st));
        AW_CUDA(B->h_packed.ensure(4 * (size_t)total));
        AW_CUDA(cudaMemcpyAsync(B->h_packed.p, B->packed.p, 4 * (size_t)total, cudaMemcpyDeviceToHost, B->st));
        AW_CUDA(cudaStreamSynchronize(B->st));
    }
    const uint32_t *hp = B->h_packed.as<uint32_t>();
    int rc = AW_OK;
    for (int i = 0; i < n; ++i) {
        ksw_extz_t *z = &ez[i];
        reset_extz(z);
        if (pl->early_zdrop[i]) { z->zdropped = 1; continue; }
        if (!pl->route[i]) continue;
        const KswOut &o = ho[i];
        z->max = (uint32_t)o.max & 0x7fffffffu;
        z->max_q = o.max_q, z->max_t = o.max_t, z->mqe = o.mqe, z->mqe_t = o.mqe_t;
        z->mte = o.mte, z->mte_q = o.mte_q, z->score = o.score;
        z->zdropped = o.zdropped ? 1 : 0, z->reach_end = o.reach_end, z->stopped = o.stopped;
        if (cigar && o.n_cigar > 0) {
            if (!store_cigar(km, z, hp + poff[i], o.n_cigar)) { z->zdropped = 1; rc = AW_E_NOMEM; }
        }
    }
    return rc;
}

// ---- exported entry points --------------------------------------------------------------
extern "C" {

const char *aw_last_error(void) { return tls_err.c_str(); }

int aw_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

void aw_set_traceback_budget(int64_t bytes) {
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    g_tb_budget = bytes;
}

void aw_release_thread_buffers(void) {
    if (tls_buf) {
        delete tls_buf;
        tls_buf = nullptr;
    }
}

void aw_ksw_set_deadline(double seconds) {
    if (seconds > 0.0 && seconds < 1e9) {
        tls_has_deadline = true;
        tls_deadline = std::chrono::steady_clock::now() +
                       std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                           std::chrono::duration<double>(seconds));
    } else {
        tls_has_deadline = false;
    }
}

void aw_ksw_set_stop_antidiagonal(int interval, int antidiagonal) { set_exact_stop(interval, antidiagonal); }

void aw_set_full_pair_routing(int enabled) { g_band_full_pairs.store(enabled != 0); }

void aw_set_band_columns(int columns) {
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    g_band_nc = (columns == 4 || columns == 8) ? columns : 0;
}

void aw_set_tuning(int large_warps, int large_tlen_threshold) {
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    if (large_warps == 1 || large_warps == 2 || large_warps == 4 || large_warps == 8) g_large_warps = large_warps;
    if (large_tlen_threshold > 0) g_large_tlen = large_tlen_threshold;
}

aw_ksw_plan_t *aw_ksw_plan_new(int n, const int *qlen, const int *tlen, const int *w, int8_t m,
                               const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2, int zdrop,
                               int end_bonus, int flag) {
    if (n < 0 || (n > 0 && (!qlen || !tlen || !mat))) { set_error("invalid arguments"); return nullptr; }
    aw_ksw_plan_t *pl = new aw_ksw_plan_t();
    pl->B = &pl->own;
    if (!make_params(m, mat, q, e, q2, e2, zdrop, end_bonus, flag, pl->P)) {
        set_error("alphabet size m must be 2..8");
        delete pl;
        return nullptr;
    }
    if (plan_build(pl, n, qlen, tlen, w) || plan_alloc(pl)) { delete pl; return nullptr; }
    return pl;
}

int aw_ksw_plan_upload(aw_ksw_plan_t *pl, const uint8_t *const *query, const uint8_t *const *target) {
    if (!pl) return AW_E_INVAL;
    return plan_upload(pl, query, target);
}

// Plans above this many DP cells (about 20 ms of device work) always launch eagerly.
static constexpr int64_t kGraphMaxCells = 20000000000LL;

int aw_ksw_plan_execute(aw_ksw_plan_t *pl, float *ms) {
    if (!pl) return AW_E_INVAL;
    pl->graph_used = false;
    // graphs for the strip and banded kernels of plans small enough that launch overhead
    // matters (on the 4,096-pair bench plan, 1.7e11 cells, replaying the graph measured 5-8%
    // slower than launching eagerly); the anti-diagonal kernel synchronises on the host
    // between workspace groups, and a deadline is re-armed per call
    if (pl->graph_off || !pl->uploaded || !pl->exact_ids.empty() || tls_has_deadline ||
        pl->cells > kGraphMaxCells)
        return plan_execute(pl, ms);
    int lw;
    {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        lw = g_large_warps;
    }
    if (pl->gexec && pl->graph_warps != lw) pl->drop_graph();  // tuning changed: capture again
    if (!pl->gexec) {
        if (pl->eager_runs < 1) {
            ++pl->eager_runs;
            return plan_execute(pl, ms);
        }
        Buffers *B = pl->B;
        AW_CUDA(cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal));
        tls_capturing = true;
        const int rc = plan_launch(pl);
        tls_capturing = false;
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(B->st, &g);
        cudaGraphExec_t ge = nullptr;
        if (rc || ec != cudaSuccess || !g || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
            // a step of this plan cannot be captured here: keep running it eagerly
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            pl->graph_off = true;
            return plan_execute(pl, ms);
        }
        pl->graph = g, pl->gexec = ge, pl->graph_warps = lw;
    }
    AW_CUDA(cudaGraphLaunch(pl->gexec, pl->B->st));
    pl->graph_used = true;
    return plan_finish(pl, ms);
}

int aw_ksw_plan_graph(const aw_ksw_plan_t *pl) { return pl && pl->graph_used ? 1 : 0; }

int aw_ksw_plan_download(aw_ksw_plan_t *pl, ksw_extz_t *ez) {
    if (!pl || !ez) return AW_E_INVAL;
    return plan_download(pl, ez, nullptr);
}

int aw_ksw_plan_stats(const aw_ksw_plan_t *pl, int64_t *cells, int64_t *tb_bytes, int *waves, int *launches) {
    if (!pl) return AW_E_INVAL;
    if (cells) *cells = pl->cells;
    if (tb_bytes) *tb_bytes = pl->tb_total;
    if (waves) *waves = (int)pl->waves.size();
    if (launches) *launches = pl->launches;
    return AW_OK;
}

int aw_ksw_plan_routes(const aw_ksw_plan_t *pl, int *strip_pairs, int *banded_pairs, int *exact_pairs) {
    if (!pl) return AW_E_INVAL;
    int n[4] = {0, 0, 0, 0};
    for (int r : pl->route) ++n[r];
    if (strip_pairs) *strip_pairs = n[1];
    if (banded_pairs) *banded_pairs = n[3];
    if (exact_pairs) *exact_pairs = n[2];
    return AW_OK;
}

int aw_ksw_plan_timing(const aw_ksw_plan_t *pl, float *dp_ms, float *bt_ms) {
    if (!pl) return AW_E_INVAL;
    if (dp_ms) *dp_ms = pl->dp_ms;
    if (bt_ms) *bt_ms = pl->bt_ms;
    return AW_OK;
}

void aw_ksw_plan_free(aw_ksw_plan_t *pl) { delete pl; }

int aw_ksw_extd2_batch(int n, const int *qlen, const uint8_t *const *query, const int *tlen,
                       const uint8_t *const *target, const int *w, int8_t m, const int8_t *mat, int8_t q,
                       int8_t e, int8_t q2, int8_t e2, int zdrop, int end_bonus, int flag, ksw_extz_t *ez) {
    if (n < 0 || (n > 0 && (!qlen || !tlen || !query || !target || !mat || !ez))) return AW_E_INVAL;
    if (n == 0) return AW_OK;
    aw_ksw_plan_t pl;
    pl.B = thread_buffers();
    if (!make_params(m, mat, q, e, q2, e2, zdrop, end_bonus, flag, pl.P)) {
        set_error("alphabet size m must be 2..8");
        for (int i = 0; i < n; ++i) reset_extz(&ez[i]), ez[i].zdropped = 1;
        return AW_E_UNSUPPORTED;
    }
    int rc = plan_build(&pl, n, qlen, tlen, w);
    if (!rc) rc = plan_alloc(&pl);
    if (!rc) rc = plan_upload(&pl, query, target);
    if (!rc) rc = plan_execute(&pl, nullptr);
    if (!rc) rc = plan_download(&pl, ez, nullptr);
    if (rc)
        for (int i = 0; i < n; ++i)
            if (!pl.executed) reset_extz(&ez[i]), ez[i].zdropped = 1;
    pl.B = nullptr;
    return rc;
}

static void single_call(void *km, int qlen, const uint8_t *query, int tlen, const uint8_t *target, int8_t m,
                        const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2, int w, int zdrop,
                        int end_bonus, int flag, ksw_extz_t *ez) {
    reset_extz(ez);
    if (m <= 1 || qlen <= 0 || tlen <= 0) return;
    aw_ksw_plan_t pl;
    pl.B = thread_buffers();
    if (!make_params(m, mat, q, e, q2, e2, zdrop, end_bonus, flag, pl.P)) {
        set_error("alphabet size m must be 2..8");
        ez->zdropped = 1;
        return;
    }
    // one pair alone: let a whole warp group pipeline its strips whatever its length
    tls_all_large = true;
    int rc = plan_build(&pl, 1, &qlen, &tlen, &w);
    tls_all_large = false;
    if (!rc) rc = plan_alloc(&pl);
    if (!rc) rc = plan_upload(&pl, &query, &target);
    if (!rc) rc = plan_execute(&pl, nullptr);
    if (!rc) rc = plan_download(&pl, ez, km);
    if (rc && !pl.executed) reset_extz(ez), ez->zdropped = 1;
    pl.B = nullptr;
}

void ksw_extd2_gpu(void *km, int qlen, const uint8_t *query, int tlen, const uint8_t *target, int8_t m,
                   const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2, int w, int zdrop,
                   int end_bonus, int flag, ksw_extz_t *ez) {
    single_call(km, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus,
                flag & ~(AW_EZ_SINGLETRACK | AW_EZ_SSE_SINGLETRACK), ez);
}

void ksw_extd2_singletrack_gpu(void *km, int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                               int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2, int w,
                               int zdrop, int end_bonus, int flag, ksw_extz_t *ez) {
    single_call(km, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus,
                (flag | AW_EZ_SINGLETRACK) & ~AW_EZ_SSE_SINGLETRACK, ez);
}

void ksw_extd2_singletrack_sse_gpu(void *km, int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                                   int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2, int w,
                                   int zdrop, int end_bonus, int flag, ksw_extz_t *ez) {
    single_call(km, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus,
                flag | AW_EZ_SINGLETRACK | AW_EZ_SSE_SINGLETRACK, ez);
}

}  // extern "C"

namespace aw {
// Traceback budget of the calling thread's batches (0 = the process-wide setting).
void set_thread_tb_budget(int64_t bytes) { tls_tb_budget = bytes; }

// Allocates the calling thread's traceback arena up front (serving workers), so that
// batches do not grow it (a device-wide synchronisation) while other workers run.
int reserve_thread_tb(int64_t bytes) {
    Buffers *B = thread_buffers();
    if (B->init()) return AW_E_CUDA;
    return B->tb.ensure((size_t)bytes + 256) == cudaSuccess ? AW_OK : AW_E_CUDA;
}

// Parameter checks and score table of the full-matrix strip path, for callers
// outside this file.  Returns AW_OK when (qlen, tlen, parameters, flag) can run
// on the strip kernel, 1 when ksw_extd2 would return at once without any DP
// (the ksw2_extd2_sse.c:81/:105 early exits), AW_E_UNSUPPORTED otherwise.
int full_path_params(int qlen, int tlen, int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2,
                     int8_t e2, int flag, KswScore *S) {
    if (m <= 1 || qlen <= 0 || tlen <= 0) return 1;
    Params P;
    if (!make_params(m, mat, q, e, q2, e2, -1, 0, flag, P)) return AW_E_UNSUPPORTED;
    if (P.early_return) return 1;
    if (!full_path_ok(P, qlen, tlen, -1)) return AW_E_UNSUPPORTED;
    *S = make_score(P);
    return AW_OK;
}
}  // namespace aw
