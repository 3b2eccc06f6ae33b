/*
 * anchorwave_b200.h -- C ABI of libaw_b200.so, the B200 (sm_100a) implementation
 * of AnchorWave's per-interval alignment kernels.
 *
 * Plain C types only (pointers, sizes, ints); no CUDA or torch types.  Every
 * entry point is reentrant: each host thread gets its own CUDA stream and its
 * own pooled device buffers.  Errors never cross the ABI as exceptions; the
 * drop-in KSW2 entries report them as ez->zdropped = 1 (the reference's own
 * failure convention, minimap2/ksw2_extd2_avx.c:138-141) and record a message
 * readable with aw_last_error().
 */
#ifndef ANCHORWAVE_B200_H
#define ANCHORWAVE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef KSW2_H_
/* Result record, layout-identical to ksw_extz_t of minimap2/ksw2.h:40-50. */
typedef struct {
    uint32_t max:31, zdropped:1;
    int max_q, max_t;      /* max extension coordinate */
    int mqe, mqe_t;        /* max score when reaching the end of query */
    int mte, mte_q;        /* max score when reaching the end of target */
    int score;             /* max score reaching both ends; may be KSW_NEG_INF */
    int m_cigar, n_cigar;
    int reach_end;
    int stopped;           /* cooperative stop requested */
    uint32_t *cigar;       /* BAM ops: len<<4 | {0=M,1=I,2=D} */
} ksw_extz_t;
#endif

/* ---- drop-in KSW2 entries -------------------------------------------------- */

/*
 * Replaces ksw_extd2_sse / ksw_extd2_avx2 / ksw_extd2_avx512
 * (minimap2/ksw2.h:91-107; called from
 * src/myImportandFunction/alignSlidingWindow.cpp:288-297, :380-389, :762-792,
 * :840-846).  Same arguments, same ksw_extz_t results bit for bit (scores, end
 * coordinates, CIGAR including tie-breaking) as the AVX-512 kernel.
 * CIGAR ownership as in the reference: the buffer is (re)allocated with
 * krealloc(km, ...) when km != NULL (kalloc arena of the calling process,
 * looked up at run time) and with realloc() when km == NULL; the caller frees
 * it with kfree(km, ez->cigar) / free().  ez->m_cigar/ez->cigar on entry are
 * reused like ksw_push_cigar does.
 */
void ksw_extd2_gpu(void *km, int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                   int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                   int w, int zdrop, int end_bonus, int flag, ksw_extz_t *ez);

/*
 * Replaces ksw_extd2_singletrack_avx512 / _avx2 (minimap2/ksw2_singletrack.hpp:32-46):
 * KSW2 score recurrence with the Singletrack two-track traceback.
 */
void ksw_extd2_singletrack_gpu(void *km, int qlen, const uint8_t *query, int tlen,
                               const uint8_t *target, int8_t m, const int8_t *mat, int8_t q,
                               int8_t e, int8_t q2, int8_t e2, int w, int zdrop, int end_bonus,
                               int flag, ksw_extz_t *ez);

/*
 * Replaces ksw_extd2_singletrack_sse (minimap2/ksw2_singletrack.hpp:17-32;
 * ksw2_singletrack.cpp:202-626), the Singletrack entry of builds without AVX2
 * (alignSlidingWindow.cpp:942-948): 16-byte-block band semantics, mqe/mte on a strict
 * ">", mte_q = r - en with en rounded up to its block, and the reconstruction whatever the
 * EXTZ/SEMIGLOBAL flags.  Same signature; the batch entries take the same behaviour from
 * flag AW_EZ_SINGLETRACK | AW_EZ_SSE_SINGLETRACK.
 */
void ksw_extd2_singletrack_sse_gpu(void *km, int qlen, const uint8_t *query, int tlen,
                                   const uint8_t *target, int8_t m, const int8_t *mat, int8_t q,
                                   int8_t e, int8_t q2, int8_t e2, int w, int zdrop, int end_bonus,
                                   int flag, ksw_extz_t *ez);
#define AW_EZ_SINGLETRACK     0x1000  /* flag: the Singletrack traceback */
#define AW_EZ_SSE_SINGLETRACK 0x4000  /* flag, with AW_EZ_SINGLETRACK: as ksw_extd2_singletrack_sse */

/* ---- batched KSW2 ------------------------------------------------------------ */

/*
 * n independent ksw_extd2 calls in one submission (the batched form of the
 * AnchorTaskExecutor loop, src/service/AnchorTaskExecutor.h:54-160).  Pair i
 * is (query[i], qlen[i]) x (target[i], tlen[i]) with band w[i] (w == NULL:
 * all -1).  Results land in ez[i] exactly as n calls of ksw_extd2_gpu would
 * leave them; ez[i].cigar is malloc'd (km semantics: NULL arena).
 * Returns 0 on success, a negative AW_E* code otherwise.
 */
int aw_ksw_extd2_batch(int n, const int *qlen, const uint8_t *const *query, const int *tlen,
                       const uint8_t *const *target, const int *w, int8_t m, const int8_t *mat,
                       int8_t q, int8_t e, int8_t q2, int8_t e2, int zdrop, int end_bonus,
                       int flag, ksw_extz_t *ez);

/* Plan API: keep a batch resident on the device to run it repeatedly. */
typedef struct aw_ksw_plan aw_ksw_plan_t;
aw_ksw_plan_t *aw_ksw_plan_new(int n, const int *qlen, const int *tlen, const int *w, int8_t m,
                               const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                               int zdrop, int end_bonus, int flag);
int aw_ksw_plan_upload(aw_ksw_plan_t *plan, const uint8_t *const *query,
                       const uint8_t *const *target);
/* Runs every wave of the plan on its stream; ms (optional) receives the CUDA-event
 * time of the device work between the first and the last launch. */
int aw_ksw_plan_execute(aw_ksw_plan_t *plan, float *ms);
/* 1 when the last aw_ksw_plan_execute replayed the plan as a CUDA graph.  For plans of
 * up to 2e10 DP cells (where launch overhead is a visible part of an execute) the first
 * execute runs eagerly, the second captures the launch sequence into a graph, later ones
 * replay it (one launch call per execute).  Larger plans, plans with pairs on the
 * anti-diagonal kernel (z-drop, approximate max, extension-only, positive match scores)
 * and executes under a deadline (aw_ksw_set_deadline) always launch eagerly.  No
 * counterpart in the reference (its calls are one-shot). */
int aw_ksw_plan_graph(const aw_ksw_plan_t *plan);
int aw_ksw_plan_download(aw_ksw_plan_t *plan, ksw_extz_t *ez);
/* Device-side statistics of the plan: cells, traceback bytes, waves, launches. */
int aw_ksw_plan_stats(const aw_ksw_plan_t *plan, int64_t *cells, int64_t *tb_bytes, int *waves,
                      int *launches_per_execute);
/* How the plan routes its pairs: the full-matrix strip kernel, the banded strip kernel
 * (banded calls, Singletrack calls of either entry, long full-width pairs) and the exact
 * anti-diagonal kernel (z-drop, approximate max, extension-only, parameters beyond the
 * strip kernels' magnitude bound).  Pairs with no device work count in none. */
int aw_ksw_plan_routes(const aw_ksw_plan_t *plan, int *strip_pairs, int *banded_pairs, int *exact_pairs);
/* CUDA-event times (ms) of the last execute, summed over waves: the DP phase (the
 * concurrent strip-kernel launches) and the traceback phase (backtrack kernel). */
int aw_ksw_plan_timing(const aw_ksw_plan_t *plan, float *dp_ms, float *bt_ms);
void aw_ksw_plan_free(aw_ksw_plan_t *plan);

/* Gapped alignment rows from KSW2 CIGARs, decoded on the device: the rows AnchorWave's
 * callers build on the host before the MAF writer (src/myImportandFunction/
 * alignSlidingWindow.cpp:307-324).  Pair i: CIGAR cigar[i][0..n_cigar[i]) over query[i]
 * (qlen[i] characters) and target[i] (tlen[i]); row_q / row_d receive the aligned query and
 * reference back to back, pair i at row_off[i] with row_len[i] characters (capacity: room
 * in each row buffer).  M, = and X copy both sequences, I copies the query against '-', D
 * puts '-' against the reference.  Returns 0, or AW_E_INVAL for another operation, a CIGAR
 * that runs past the end of a sequence, or rows beyond the capacity. */
int aw_cigar_rows_batch(int n, const uint32_t *const *cigar, const int *n_cigar, const char *const *query,
                        const int *qlen, const char *const *target, const int *tlen, char *row_q, char *row_d,
                        int64_t *row_off, int *row_len, int64_t capacity);

/* ---- rescue procedures (batched) ---------------------------------------------- */

/* Result of alignScoreCertifiedKsw2 (src/myImportandFunction/alignSlidingWindow.h:31-49:
 * Ksw2CertifiedStatus and Ksw2CertifiedResult) for one interval.  status: 0 Completed,
 * 1 TimeLimit, 2 NotCertified, 3 Failed.  alignment_q/_d: the certified rows (malloc'd,
 * NUL-terminated, alignment_len characters), only when Completed; best_effort_q/_d: the
 * best valid banded rows of a failed certification.  Free with aw_certified_result_free. */
typedef struct {
    int status;
    int64_t score, optimal_score, final_band_width, traceback_attempts;
    char *alignment_q, *alignment_d;
    int64_t alignment_len;
    char *best_effort_q, *best_effort_d;
    int64_t best_effort_len;
} aw_certified_result_t;

/*
 * alignScoreCertifiedKsw2 (src/myImportandFunction/alignSlidingWindow.cpp:1197-1400) for n
 * intervals at once, called from the executor at :1835: the unbanded score-only optimum of
 * every interval in one batch, then round by round the next band of every interval not yet
 * certified in one banded batch, until its re-scored alignment reaches the optimum; the
 * skipped smallest band runs only on failure.  Untimed calls let a round take an interval's
 * next few bands (up to 4e9 band cells together) and fold their results in band order, so
 * the narrow bands of a long interval, each bound by its strip chain, cost one round.  Every interval gets the result a call of its
 * own would give (the selector's chained traceback, used when a selection plan is passed,
 * stays with the caller).  Sequences are ASCII; initial_band_width / maximum_band_width hold
 * interval i's bands (the selection plan's ksw2CertifiedInitialBandWidth and
 * ksw2CertifiedMaximumBandWidth); penalties AnchorWave's (negative); maximum_runtime_seconds
 * > 0 arms the calling thread's deadline (aw_ksw_set_deadline) for the call;
 * precomputed_optimal_scores (n values, or NULL) skips the score-only batch.  Returns AW_OK
 * or a negative AW_E* code; out[i] is filled either way.
 */
int aw_align_score_certified_batch(int n, const char *const *query, const int64_t *qlen,
                                   const char *const *reference, const int64_t *rlen,
                                   const int64_t *initial_band_width, const int64_t *maximum_band_width,
                                   int32_t mismatching_penalty, int32_t open1, int32_t extend1, int32_t open2,
                                   int32_t extend2, double maximum_runtime_seconds,
                                   const int64_t *precomputed_optimal_scores, aw_certified_result_t *out);
void aw_certified_result_free(aw_certified_result_t *result);

/* Result of the sliding-window alignment: the whole alignment's two-piece affine score and
 * its rows (malloc'd, NUL-terminated).  Free with aw_window_result_free. */
typedef struct {
    int64_t score;
    char *alignment_q, *alignment_d;
    int64_t alignment_len;
} aw_window_result_t;

/*
 * alignSlidingWindow (src/myImportandFunction/alignSlidingWindow.cpp:457-590), the
 * approximate-tier fallback called from the executor at :2683, for n intervals at once: an
 * interval with (rlen/W)*(qlen/W) <= 1 gets one global alignment (W = window[i], e.g. the
 * selection plan's slidingWindowWidth); the others advance window by window (W+1 bases of
 * each sequence, semiglobal KSW2 ending at the better of the last row and the last column),
 * the k-th window of every interval still advancing in one batched call; trailing gaps close
 * the alignment, which is re-scored with the two-piece objective.  Sequences ASCII,
 * penalties negative.  Returns AW_OK or a negative AW_E* code (an endpoint the traceback
 * does not reconstruct is AW_E_INVAL, the reference's runtime_error).
 */
int aw_align_sliding_window_batch(int n, const char *const *query, const int64_t *qlen,
                                  const char *const *reference, const int64_t *rlen, const int64_t *window,
                                  int32_t matching_score, int32_t mismatching_penalty, int32_t open1,
                                  int32_t extend1, int32_t open2, int32_t extend2, aw_window_result_t *out);
void aw_window_result_free(aw_window_result_t *result);

/* ---- WFA (gap-affine-2p, end to end) ------------------------------------------ */

/* Attributes of WfaAlignment.cpp:143-170: match 0, these penalties (positive), no
 * heuristic, full CIGAR; memory_mode as WFA2-lib's wavefront_memory_t
 * (wavefront/wavefront_attributes.h:122-127): 0 high (every wavefront kept), 1 medium and
 * 2 low (piggyback: a ring of recent scores plus packed-CIGAR blocks; the ultralow
 * BiWFA mode 3 is not provided).  singletrack selects the Singletrack traceback and, as in
 * wavefront/wavefront_aligner.c:251-260, only applies in high memory. */
typedef struct {
    int mismatch, gap_opening1, gap_extension1, gap_opening2, gap_extension2;
    int singletrack;
    int memory_mode;
    int64_t max_memory_abort;   /* device pool cap in bytes (0 = 85% of free memory) */
} wavefront_gpu_attr_t;

typedef struct wavefront_aligner_gpu wavefront_aligner_gpu_t;

/* Replaces wavefront_aligner_new (WFA2-lib wavefront/wfa.h:129-134). */
wavefront_aligner_gpu_t *wavefront_aligner_new_gpu(const wavefront_gpu_attr_t *attr);
/* Replaces wavefront_aligner_delete. */
void wavefront_aligner_delete_gpu(wavefront_aligner_gpu_t *aligner);
/* Replaces wavefront_align (wfa.h:210-215): pattern = reference, text = query.
 * Returns the WF status (0 completed, -200 out of memory, -300 unattainable). */
int wavefront_align_gpu(wavefront_aligner_gpu_t *aligner, const char *pattern, int pattern_length,
                        const char *text, int text_length);
/* The last alignment's CIGAR operations ('M','X','I','D'; the aligner->cigar
 * operations[begin_offset..end_offset) of the reference) and its score (-penalty). */
int wavefront_gpu_cigar(const wavefront_aligner_gpu_t *aligner, const char **operations,
                        int *num_operations, int *score);
/* n alignments in one submission.  ops (capacity >= sum(plen + tlen) bytes) receives
 * the operations back to back, pair i at ops_offset[i] with n_ops[i] characters. */
int wavefront_align_batch_gpu(wavefront_aligner_gpu_t *aligner, int n, const char *const *pattern,
                              const int *pattern_length, const char *const *text,
                              const int *text_length, int *status, int *score,
                              int64_t *ops_offset, int *n_ops, char *ops, int64_t ops_capacity,
                              float *device_ms);
/* Device memory the last call's alignments took from the wavefront pool (headers,
 * wavefronts and packed-CIGAR blocks; the reference's align_status.memory_used,
 * WfaAlignment.cpp:353-354): the largest single alignment and the sum over the call. */
int wavefront_gpu_memory(const wavefront_aligner_gpu_t *aligner, int64_t *pair_max, int64_t *total);
/* High memory (standard and Singletrack): a pair whose wavefront grows wider than `width`
 * diagonals, or wider than `tail_width` once every pair of the call has started and no more
 * pairs run on warps than clusters fit on the device (the call's tail), leaves its
 * warp and runs again from score 0 on a cluster of `cluster_ctas` CTAs (1..8) that spreads
 * each wavefront over all of their threads; results are identical.  width 0: every pair
 * stays on one warp; a negative value or cluster_ctas <= 0 keeps that setting.  Defaults:
 * 8192, 1024 and 8.  Process-wide.  No counterpart in the reference (tuning knob). */
void aw_set_wfa_wide(int width, int tail_width, int cluster_ctas);
/* High memory: pairs whose pattern and text lengths sum to at least `min_length_sum` run
 * first, each on all four warps of a CTA (the longest pairs of a batch otherwise set its
 * duration, one warp each); the others then run one per warp.  0: every pair starts on one
 * warp.  Default 1536.  A CTA's pair moves to the cluster kernel by the widths of
 * aw_set_wfa_wide, as a warp's does.  Results are identical.  Process-wide. */
void aw_set_wfa_long(int min_length_sum);
/* Kernel launches of the last call (every round and phase) and, of them, the cluster
 * kernel's, with the number of pairs that moved to it. */
int wavefront_gpu_last_launches(const wavefront_aligner_gpu_t *aligner, int *launches, int *cluster_launches,
                                int *cluster_pairs);

/* ---- selector sequence summary ------------------------------------------------- */

/* One sequence of summarizeSequencePair (src/myImportandFunction/
 * AlignmentAlgorithmSelector.cpp:180-191, :730-757): FNV-1a fingerprint, the fraction of
 * bases other than A/C/G/T, the mean normalized entropy of 64-base blocks, the fraction
 * of bases at run length >= 4, and the k = 9, 15, 21 sketches (hash, start position;
 * position order, at most 4 entries per hash) at sketch_offset[s], sketch_count[s]
 * entries, in the arrays of aw_sequence_summary_sketches. */
typedef struct {
    uint64_t fingerprint;
    double ambiguous_fraction, normalized_entropy, low_complexity_fraction;
    int64_t sketch_offset[3];
    int64_t sketch_count[3];
} aw_sequence_summary_t;

/* Replaces summarizeSequencePair for n interval pairs on the device: out[2i] = query i,
 * out[2i+1] = reference i, identical[i] = the two are equal.  modulos: n x 3 sampling
 * modulos, or NULL for those of makeAlignmentSelectionPlan (:1752-1760).  The sketches
 * stay with the calling thread until its next call.  Returns 0 or a negative AW_E_*. */
int aw_sequence_summary_batch(int n, const char *const *query, const int64_t *qlen,
                              const char *const *reference, const int64_t *rlen,
                              const uint64_t *modulos, aw_sequence_summary_t *out, int *identical,
                              float *device_ms);
/* Copies the calling thread's last sketches (capacity entries at least; hash and position
 * both NULL: returns the number of entries only).  Returns the number of entries. */
int64_t aw_sequence_summary_sketches(uint64_t *hash, uint32_t *position, int64_t capacity);
/* The same entries without a copy: pointers into the calling thread's page-locked
 * buffers, valid until its next aw_sequence_summary_batch.  Returns the number of entries. */
int64_t aw_sequence_summary_sketch_view(const uint64_t **hash, const uint32_t **position);

/* ---- serving loop (continuous batching) --------------------------------------- */

/* Engine of a request, as chosen by AnchorWave's exact-tier / fallback-tier selector
 * (src/myImportandFunction/AlignmentAlgorithmSelector.cpp:1711). */
#define AW_ROUTE_KSW2             0  /* ksw_extd2, full (band < 0) or banded */
#define AW_ROUTE_KSW2_SINGLETRACK 1  /* ksw_extd2 with the Singletrack traceback */
#define AW_ROUTE_WFA              2  /* gap-affine-2p WFA, high memory */
#define AW_ROUTE_WFA_SINGLETRACK  3  /* gap-affine-2p WFA, Singletrack */
#define AW_ROUTE_WFA_MEDIUM       4  /* gap-affine-2p WFA, medium memory (piggyback) */
#define AW_ROUTE_WFA_LOW          5  /* gap-affine-2p WFA, low memory (piggyback) */
#define AW_ROUTE_KSW2_CERTIFIED   6  /* score-certified KSW2 (aw_align_score_certified_batch) */
#define AW_ROUTE_SLIDING_WINDOW   7  /* sliding-window semiglobal KSW2 (aw_align_sliding_window_batch) */

/* A request's engine and its parameters, as the selection plan gives them
 * (src/myImportandFunction/AlignmentAlgorithmSelector.h:196-242): band (KSW2 band width, -1
 * = full; the initial band of score-certified KSW2), band_max (score-certified KSW2's largest
 * band), window (the sliding-window width) and predicted_bytes (the plan's memoryBytes
 * estimate of the engine, AlignmentAlgorithmSelector.h:87; 0 = the server's own estimate),
 * which the server uses for admission and to keep a WFA micro-batch within its wavefront
 * pool. */
typedef struct {
    int method;
    int band;
    int band_max;
    int64_t window;
    int64_t predicted_bytes;
} aw_serve_route_t;

typedef struct {
    int slots;            /* concurrent micro-batches (workers with their own streams) */
    int max_batch;        /* requests per micro-batch */
    int64_t hbm_budget;   /* device bytes of the server: admission of predicted bytes, and the
                             pooled buffers of its workers (0 = 70% of free memory) */
    int8_t m;             /* KSW2 scoring: alphabet size, m*m matrix, q, e, q2, e2 */
    int8_t mat[64];
    int8_t q, e, q2, e2;
    int wfa_x, wfa_o1, wfa_e1, wfa_o2, wfa_e2;  /* WFA penalties (positive) */
} aw_serve_config_t;

typedef struct {
    uint64_t id;
    int method;
    int status;           /* 0 ok; WF status for WFA routes; AW_E* on failure; for score-certified
                             KSW2 the certification status (0 Completed, 1 TimeLimit,
                             2 NotCertified, 3 Failed) */
    ksw_extz_t ez;        /* KSW2 routes: ez.cigar malloc'd.  Score-certified and sliding-window
                             routes: the rows as a CIGAR (M/I/D) and ez.score = their re-scored
                             two-piece score (a failed certification: its best-effort rows) */
    int wfa_score;        /* WFA routes: -penalty */
    int n_ops;
    char *ops;            /* WFA routes: 'M','X','I','D' operations, malloc'd */
    double latency_s;     /* submit -> result ready */
} aw_serve_result_t;

typedef struct {
    uint64_t submitted, completed, micro_batches, queued;
    int64_t inflight_bytes;
    double latency_p50_s, latency_p99_s, elapsed_s;
} aw_serve_stats_t;

typedef struct aw_server aw_server_t;

/* Replaces the alignment-stage thread pool (src/service/AnchorTaskExecutor.h:54-160). */
aw_server_t *aw_serve_open(const aw_serve_config_t *cfg);
/* Enqueue one interval (ASCII sequences; ids consecutive from 0). Never blocks on the GPU. */
int aw_serve_submit(aw_server_t *server, uint64_t id, int method, int band, const char *query,
                    int qlen, const char *target, int tlen);
/* The same with every parameter of the route (required for AW_ROUTE_KSW2_CERTIFIED and
 * AW_ROUTE_SLIDING_WINDOW; aw_serve_submit leaves band_max = -1 and window = 0). */
int aw_serve_submit_route(aw_server_t *server, uint64_t id, const aw_serve_route_t *route, const char *query,
                          int qlen, const char *target, int tlen);
/* Up to max finished results, strictly in id order (waits up to wait_ms for the next one). */
int aw_serve_poll(aw_server_t *server, aw_serve_result_t *out, int max, int wait_ms);
int aw_serve_stats(aw_server_t *server, aw_serve_stats_t *stats);
void aw_serve_result_free(aw_serve_result_t *result);
void aw_serve_close(aw_server_t *server);

/* ---- allocation-free entry (no counterpart in the reference) ----------------------- */

/* Scalar ksw_extz_t fields as written to device memory by the entry below. */
typedef struct {
    int32_t score, max, max_q, max_t, mqe, mqe_t, mte, mte_q;
    int32_t n_cigar, zdropped, reach_end, stopped;
} aw_ksw_result_t;

/* Size of the fixed device scratch array behind aw_ksw_extd2_device_noalloc. */
#define AW_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/*
 * Full-matrix global ksw_extd2 (w = -1, no z-drop) of one pair, for callers that
 * must not allocate device memory at call time: a process whose device memory is
 * entirely reserved by its own caching allocator, or a latency-critical loop that
 * cannot take the implicit synchronisation of cudaMalloc/cudaFree.  This entry
 * point has no counterpart in the reference.  All buffers are the caller's device
 * memory: d_query/d_target hold 0..m-1 codes, *d_result receives the scalar
 * fields and d_cigar (cigar_capacity >= qlen + tlen words; may be NULL with
 * KSW_EZ_SCORE_ONLY) the CIGAR, both exactly as ksw_extd2_gpu would produce.
 * mat stays in host memory.  Work is enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream); the call returns without waiting.
 * Scratch comes from one fixed __device__ array of AW_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit; pairs whose traceback and
 * strip-boundary columns do not fit it (about 5,600 x 5,600 cells) are rejected
 * with AW_E_NOMEM.  Calls share that array: calls whose GPU work overlaps race
 * and must be serialised by the caller.  The first call on a device resolves the
 * array's address (cudaGetSymbolAddress), so make it before any stream capture;
 * the address is kept until exit, so do not reset the device between calls.
 * Flags beyond SCORE_ONLY / RIGHT / GENERIC_SC / REV_CIGAR / SEMIGLOBAL_END, and
 * parameters outside the strip kernel's exact int8 envelope, return
 * AW_E_UNSUPPORTED, and so does a deterministic stop set on the calling thread
 * (aw_ksw_set_stop_antidiagonal); the thread's deadline (aw_ksw_set_deadline) is
 * not applied.  The full-matrix path never z-drops, so d_result->zdropped = 1
 * (with n_cigar = 0) means that a bounded wait between the cooperating warps gave
 * up; the call itself has already returned AW_OK by then, as the work is only
 * enqueued.  Returns AW_OK or a negative AW_E* code (aw_last_error()).
 */
int aw_ksw_extd2_device_noalloc(int qlen, const uint8_t *d_query, int tlen, const uint8_t *d_target,
                                int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                                int flag, aw_ksw_result_t *d_result, uint32_t *d_cigar,
                                int cigar_capacity, void *stream);

/* ---- configuration and diagnostics ------------------------------------------ */

/* HBM budget (bytes) for traceback arenas per host thread; mirrors the -M
 * admission envelope (src/myImportandFunction/AlignmentResourceScheduler.cpp:706).
 * 0 = default (60% of free device memory). */
void aw_set_traceback_budget(int64_t bytes);
/* Warps that cooperate on one pair for pairs with tlen >= threshold, and the
 * threshold (autotuner knobs; 0 keeps the current value). */
void aw_set_tuning(int large_warps, int large_tlen_threshold);
/* Target columns per lane of the banded kernel (4 or 8; 0 = chosen per batch from
 * its work and its longest pair).  No counterpart in the reference (tuning knob). */
void aw_set_band_columns(int columns);
/* 1 (default): a full-matrix pair that would be its batch's critical path (a long interval
 * alone or among short ones) runs on the banded kernel at full width, whose strip pipeline
 * spans all SMs; 0: every full-matrix pair runs on the full-matrix strip kernel.  Results
 * are identical either way.  No counterpart in the reference (tuning knob). */
void aw_set_full_pair_routing(int enabled);
/* Frees the device and pinned buffers that the calling thread's KSW2 calls keep pooled
 * between calls (they grow to the largest batch seen; the next call re-creates them).
 * No counterpart in the reference (its work arrays are per call). */
void aw_release_thread_buffers(void);
/* Cooperative stop for the calling thread's KSW2 calls (single, batched, plan
 * executions): pairs still being aligned `seconds` from now stop with ez->stopped = 1,
 * score KSW_NEG_INF and no CIGAR; seconds <= 0 clears it.  Replaces the deadline probe
 * that AnchorWave installs with ksw_set_progress_callback (ScopedKswDeadline,
 * src/myImportandFunction/alignSlidingWindow.cpp:593-640; minimap2/ksw2_progress.c:15-38),
 * which the device cannot call back into: the kernels poll a device copy of the deadline
 * every 32 rows (strip kernels) or 256 anti-diagonals (exact kernel).  The deadline
 * counts from the call; the device copy is armed when the stream reaches the work. */
void aw_ksw_set_deadline(double seconds);
/* Deterministic form of the same stop for the calling thread: as a progress callback
 * (interval `interval`) that returns 0 at the first probed anti-diagonal >= antidiagonal;
 * antidiagonal < 0 clears it.  While set, every pair runs on the anti-diagonal kernel, so
 * a stopped pair's fields and partial traceback are those of ksw_extd2 with that callback
 * (minimap2/ksw2_extd2_sse.c:136-139, :400-414). */
void aw_ksw_set_stop_antidiagonal(int interval, int antidiagonal);
const char *aw_last_error(void);
int aw_device_count(void);
/* Integer-ALU peak probe: IADD3/IMNMX-class 32-bit ops per second measured on
 * the current device (used as the roofline denominator for the DP kernels). */
double aw_int32_peak_ops(void);
/* The same probe on two 16-bit fields per register, on both integer pipes (per-field adds
 * as multiply-adds on the FMA pipe, SIMD max/min on the ALU pipe): field operations per
 * second, the denominator of the full-matrix strip kernel, which computes two cells per
 * instruction on the same two pipes.  No counterpart in the reference. */
double aw_int16x2_peak_ops(void);

#define AW_OK            0
#define AW_E_INVAL     (-1)
#define AW_E_CUDA      (-2)
#define AW_E_NOMEM     (-3)
#define AW_E_TIMEOUT   (-4)
#define AW_E_UNSUPPORTED (-5)

#ifdef __cplusplus
}
#endif
#endif /* ANCHORWAVE_B200_H */
