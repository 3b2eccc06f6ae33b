/*
 * ref_shim.c -- TEST INFRASTRUCTURE (oracle).  Thin C entry points over the
 * reference's own compiled KSW2 and WFA2 code, so the tests, the golden-vector
 * generator and bench.py's CPU-baseline arm can call the reference through
 * ctypes.  Linked only into oracle/_ref/libawref_<isa>.so; the product library
 * never links or loads it.
 *
 * Every call here goes to the reference symbol AnchorWave itself calls:
 *   KSW2 full/banded/score-only: ksw_extd2_{avx512,avx2,sse}
 *       (minimap2/ksw2.h:91-107; chosen at compile time exactly as
 *        src/myImportandFunction/alignSlidingWindow.cpp:288-297 does)
 *   KSW2-Singletrack: ksw_extd2_singletrack_{avx512,avx2,sse}
 *       (minimap2/ksw2_singletrack.hpp:17-46)
 *   WFA: wavefront_aligner_new + wavefront_align with the attributes set in
 *       src/myImportandFunction/WfaAlignment.cpp:143-170
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#include "minimap2/ksw2.h"
#include "minimap2/ksw2_singletrack.hpp"
#include "wavefront/wavefront_align.h"

/* 3 = AVX-512BW entry points, 2 = AVX2, 1 = SSE. */
int awref_isa(void) {
#if defined(__AVX512BW__)
    return 3;
#elif defined(__AVX2__)
    return 2;
#else
    return 1;
#endif
}

int awref_sizeof_extz(void) { return (int)sizeof(ksw_extz_t); }

void awref_free(void *p) { free(p); }

/* variant: 0 = native KSW2 entry, 1 = SSE KSW2 entry,
 *          2 = native Singletrack entry, 3 = SSE Singletrack entry. */
void awref_ksw_extd2(int variant, int qlen, const uint8_t *query, int tlen,
                     const uint8_t *target, int8_t m, const int8_t *mat,
                     int8_t q, int8_t e, int8_t q2, int8_t e2, int w,
                     int zdrop, int end_bonus, int flag, ksw_extz_t *ez) {
    switch (variant) {
    case 0:
#if defined(__AVX512BW__)
        ksw_extd2_avx512(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#elif defined(__AVX2__)
        ksw_extd2_avx2(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#else
        ksw_extd2_sse(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#endif
        break;
    case 1:
        ksw_extd2_sse(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
        break;
    case 2:
#if defined(__AVX512BW__)
        ksw_extd2_singletrack_avx512(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#elif defined(__AVX2__)
        ksw_extd2_singletrack_avx2(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#else
        ksw_extd2_singletrack_sse(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
#endif
        break;
    default:
        ksw_extd2_singletrack_sse(0, qlen, query, tlen, target, m, mat, q, e, q2, e2, w, zdrop, end_bonus, flag, ez);
        break;
    }
}

/* Cooperative stop (minimap2/ksw2_progress.c): stop once the probed
 * anti-diagonal reaches stop_at.  Thread-local, like the reference hook. */
static __thread int awref_stop_at = -1;
static int awref_stop_probe(void *arg, int r, int total) {
    (void)arg; (void)total;
    return r < awref_stop_at;
}
void awref_set_progress_stop(int interval, int stop_at) {
    awref_stop_at = stop_at;
    ksw_set_progress_callback(awref_stop_probe, 0, interval);
}
void awref_clear_progress(void) { ksw_clear_progress_callback(); }

/* ---- WFA ---------------------------------------------------------------- */

static wavefront_aligner_t *awref_wfa_new(int mismatch, int o1, int e1, int o2,
                                          int e2, int singletrack, int memory_mode) {
    wavefront_aligner_attr_t a = wavefront_aligner_attr_default;
    a.distance_metric = gap_affine_2p;
    a.affine2p_penalties.match = 0;
    a.affine2p_penalties.mismatch = mismatch;
    a.affine2p_penalties.gap_opening1 = o1;
    a.affine2p_penalties.gap_extension1 = e1;
    a.affine2p_penalties.gap_opening2 = o2;
    a.affine2p_penalties.gap_extension2 = e2;
    a.alignment_form.span = alignment_end2end;
    a.alignment_scope = compute_alignment;
    a.memory_mode = (wavefront_memory_t)memory_mode;
    a.singletrack = singletrack ? true : false;
    a.heuristic.strategy = wf_heuristic_none;
    a.system.verbose = 0;
    a.system.max_num_threads = 1;
    return wavefront_aligner_new(&a);
}

static int awref_wfa_run(wavefront_aligner_t *al, const char *pattern, int plen,
                         const char *text, int tlen, int *score, char *ops,
                         int ops_cap, int *n_ops) {
    int status = wavefront_align(al, pattern, plen, text, tlen);
    *score = 0;
    *n_ops = 0;
    if (status == WF_STATUS_ALG_COMPLETED) {
        cigar_t *c = al->cigar;
        int n = c->end_offset - c->begin_offset;
        *score = c->score;
        *n_ops = n;
        if (ops && n <= ops_cap) memcpy(ops, c->operations + c->begin_offset, (size_t)n);
    }
    return status;
}

/* pattern = reference, text = query (WfaAlignment.cpp:344-347). */
int awref_wfa_align(const char *pattern, int plen, const char *text, int tlen,
                    int mismatch, int o1, int e1, int o2, int e2,
                    int singletrack, int memory_mode,
                    int *score, char *ops, int ops_cap, int *n_ops) {
    wavefront_aligner_t *al = awref_wfa_new(mismatch, o1, e1, o2, e2, singletrack, memory_mode);
    if (!al) return WF_STATUS_OOM;
    int st = awref_wfa_run(al, pattern, plen, text, tlen, score, ops, ops_cap, n_ops);
    wavefront_aligner_delete(al);
    return st;
}

/* ---- Threaded batch drivers for the CPU baseline -------------------------- */

/* FNV-1a over the comparable ksw_extz_t fields and the CIGAR words, in the order
 * max, zdropped, max_q, max_t, mqe, mqe_t, mte, mte_q, score, n_cigar, reach_end,
 * stopped, cigar[0..n_cigar). */
static uint64_t awref_fnv(uint64_t h, uint32_t v) {
    for (int b = 0; b < 4; ++b) { h ^= (v >> (8 * b)) & 0xff; h *= 1099511628211ULL; }
    return h;
}
uint64_t awref_extz_hash(const ksw_extz_t *ez) {
    uint64_t h = 1469598103934665603ULL;
    uint32_t f[12] = {ez->max, ez->zdropped, (uint32_t)ez->max_q, (uint32_t)ez->max_t, (uint32_t)ez->mqe,
                      (uint32_t)ez->mqe_t, (uint32_t)ez->mte, (uint32_t)ez->mte_q, (uint32_t)ez->score,
                      (uint32_t)ez->n_cigar, (uint32_t)ez->reach_end, (uint32_t)ez->stopped};
    for (int i = 0; i < 12; ++i) h = awref_fnv(h, f[i]);
    for (int i = 0; i < ez->n_cigar; ++i) h = awref_fnv(h, ez->cigar[i]);
    return h;
}

typedef struct {
    int kind;                 /* 0 = KSW2, 1 = WFA */
    int n;
    const int *qlen, *tlen;
    const int64_t *qoff, *toff;
    const uint8_t *qbuf, *tbuf;
    const int8_t *mat;
    int q, e, q2, e2, w, flag, variant;
    int wfa_x, wfa_o1, wfa_e1, wfa_o2, wfa_e2, wfa_singletrack, wfa_memory_mode;
    int32_t *score_out, *ncig_out;
    uint64_t *hash_out;
    double *sec_out;          /* per-pair seconds of the call (optional) */
    char *ops_out;            /* WFA: operations of pair i at ops_off[i] (optional) */
    const int64_t *ops_off;
    double deadline;          /* CLOCK_MONOTONIC seconds; <= 0 disables */
    volatile int next;
    volatile int done;
} awref_batch_t;

static double awref_now(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void *awref_batch_worker(void *arg) {
    awref_batch_t *b = (awref_batch_t *)arg;
    wavefront_aligner_t *al = 0; /* thread-local aligner, WfaAlignment.cpp:217-221 */
    char *ops = 0;
    int ops_cap = 0;
    for (;;) {
        if (b->deadline > 0 && awref_now() > b->deadline) break;
        int i = __sync_fetch_and_add(&b->next, 1);
        if (i >= b->n) break;
        const uint8_t *qs = b->qbuf + b->qoff[i];
        const uint8_t *ts = b->tbuf + b->toff[i];
        if (b->kind == 0) {
            ksw_extz_t ez;
            memset(&ez, 0, sizeof(ez));
            const double t0 = b->sec_out ? awref_now() : 0;
            awref_ksw_extd2(b->variant, b->qlen[i], qs, b->tlen[i], ts, 5, b->mat,
                            (int8_t)b->q, (int8_t)b->e, (int8_t)b->q2, (int8_t)b->e2,
                            b->w, -1, 0, b->flag, &ez);
            if (b->sec_out) b->sec_out[i] = awref_now() - t0;
            if (b->score_out) b->score_out[i] = ez.score;
            if (b->ncig_out) b->ncig_out[i] = ez.n_cigar;
            if (b->hash_out) b->hash_out[i] = awref_extz_hash(&ez);
            free(ez.cigar);
        } else {
            if (!al) al = awref_wfa_new(b->wfa_x, b->wfa_o1, b->wfa_e1, b->wfa_o2,
                                        b->wfa_e2, b->wfa_singletrack, b->wfa_memory_mode);
            int need = b->qlen[i] + b->tlen[i] + 8;
            if (need > ops_cap) { free(ops); ops_cap = need; ops = (char *)malloc((size_t)ops_cap); }
            int sc = 0, nops = 0;
            const double t0 = b->sec_out ? awref_now() : 0;
            int st = awref_wfa_run(al, (const char *)ts, b->tlen[i], (const char *)qs,
                                   b->qlen[i], &sc, ops, ops_cap, &nops);
            if (b->sec_out) b->sec_out[i] = awref_now() - t0;
            if (b->score_out) b->score_out[i] = st == 0 ? sc : INT32_MIN;
            if (b->ncig_out) b->ncig_out[i] = nops;
            if (b->ops_out && st == 0) memcpy(b->ops_out + b->ops_off[i], ops, (size_t)nops);
        }
        __sync_fetch_and_add(&b->done, 1);
    }
    if (al) wavefront_aligner_delete(al);
    free(ops);
    return 0;
}

static double awref_run_batch(awref_batch_t *b, int nthreads, int *n_done) {
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    double t0 = awref_now();
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], 0, awref_batch_worker, b);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], 0);
    double t1 = awref_now();
    free(th);
    if (n_done) *n_done = b->done;
    return t1 - t0;
}

/* KSW2 over a pair list with nthreads workers pulling indices from a shared
 * counter (the AnchorTaskExecutor pattern).  Sequences are 0..4 codes packed
 * back to back; qoff/toff give each pair's start.  Stops taking new pairs after
 * time_budget_s (<= 0: no budget).  Per pair (each optional): score, n_cigar, the
 * result hash (awref_extz_hash) and the seconds of its call.  Returns wall seconds. */
double awref_ksw_batch(int n, const int *qlen, const int64_t *qoff, const uint8_t *qbuf,
                       const int *tlen, const int64_t *toff, const uint8_t *tbuf,
                       const int8_t *mat, int q, int e, int q2, int e2, int w, int flag,
                       int variant, int nthreads, double time_budget_s,
                       int32_t *score_out, int32_t *ncig_out, uint64_t *hash_out, double *sec_out,
                       int *n_done) {
    awref_batch_t b;
    memset(&b, 0, sizeof(b));
    b.kind = 0; b.n = n; b.qlen = qlen; b.tlen = tlen; b.qoff = qoff; b.toff = toff;
    b.qbuf = qbuf; b.tbuf = tbuf; b.mat = mat; b.q = q; b.e = e; b.q2 = q2; b.e2 = e2;
    b.w = w; b.flag = flag; b.variant = variant; b.score_out = score_out; b.ncig_out = ncig_out;
    b.hash_out = hash_out; b.sec_out = sec_out;
    b.deadline = time_budget_s > 0 ? awref_now() + time_budget_s : 0;
    return awref_run_batch(&b, nthreads, n_done);
}

/* WFA over a pair list (ASCII sequences; pattern = target/reference, text =
 * query), one thread-local aligner per worker (standard or Singletrack in high
 * memory, or the medium / low piggyback modes).  ops_out (optional) receives pair
 * i's CIGAR operations at ops_off[i] (room for qlen + tlen + 8 characters each). */
double awref_wfa_batch(int n, const int *qlen, const int64_t *qoff, const uint8_t *qbuf,
                       const int *tlen, const int64_t *toff, const uint8_t *tbuf,
                       int x, int o1, int e1, int o2, int e2, int singletrack, int memory_mode,
                       int nthreads, double time_budget_s,
                       int32_t *score_out, int32_t *nops_out, char *ops_out, const int64_t *ops_off,
                       int *n_done) {
    awref_batch_t b;
    memset(&b, 0, sizeof(b));
    b.kind = 1; b.n = n; b.qlen = qlen; b.tlen = tlen; b.qoff = qoff; b.toff = toff;
    b.qbuf = qbuf; b.tbuf = tbuf; b.wfa_x = x; b.wfa_o1 = o1; b.wfa_e1 = e1;
    b.wfa_o2 = o2; b.wfa_e2 = e2; b.wfa_singletrack = singletrack; b.wfa_memory_mode = memory_mode;
    b.score_out = score_out; b.ncig_out = nops_out; b.ops_out = ops_out; b.ops_off = ops_off;
    b.deadline = time_budget_s > 0 ? awref_now() + time_budget_s : 0;
    return awref_run_batch(&b, nthreads, n_done);
}
