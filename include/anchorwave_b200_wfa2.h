/*
 * anchorwave_b200_wfa2.h -- the GPU WFA aligner behind WFA2-lib's own types.
 *
 * AnchorWave builds a wavefront_aligner_attr_t from wavefront_aligner_attr_default,
 * creates an aligner with wavefront_aligner_new, aligns with wavefront_align and then
 * reads aligner->cigar (operations[begin_offset..end_offset), score) and
 * aligner->align_status.memory_used / memory_peak / memory_probe_count
 * (src/myImportandFunction/WfaAlignment.cpp:143-170, :343-356).  The entries below take
 * that same attribute struct and hand back an aligner whose members carry those names,
 * so the caller's code compiles unchanged once the three calls are renamed at its
 * compile-time switch (the same pattern as the ksw_extd2_gpu call sites).
 *
 * Types: a caller that includes WFA2-lib's headers (wavefront/wfa.h) first gets WFA2-lib's
 * own wavefront_aligner_attr_t and cigar_t, and this header only adds the GPU aligner.
 * Otherwise this header declares them itself with WFA2-lib's names, members and memory
 * layout (wavefront/wavefront_attributes.h, alignment/cigar.h, system/profiler_timer.h,
 * system/profiler_counter.h, wavefront/wavefront_heuristic.h, wavefront/wavefront_plot.h,
 * wavefront/wavefront_penalties.h, alignment/{linear,affine,affine2p}_penalties.h); the library is compiled
 * against these declarations and the tests check the layout against WFA2-lib's headers.
 */
#ifndef ANCHORWAVE_B200_WFA2_H
#define ANCHORWAVE_B200_WFA2_H

#include <stdbool.h>
#include <stdint.h>
#include <time.h>

#include "anchorwave_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef WAVEFRONT_ATTRIBUTES_H_
typedef enum { indel = 0, edit = 1, gap_linear = 2, gap_affine = 3, gap_affine_2p = 4 } distance_metric_t;
typedef enum { compute_score, compute_alignment } alignment_scope_t;
typedef enum { alignment_end2end, alignment_endsfree } alignment_span_t;
typedef struct {
    alignment_span_t span;
    bool extension;
    int pattern_begin_free, pattern_end_free, text_begin_free, text_end_free;
} alignment_form_t;
typedef struct { int match, mismatch, indel; } linear_penalties_t;
typedef struct { int match, mismatch, gap_opening, gap_extension; } affine_penalties_t;
typedef struct { int match, mismatch, gap_opening1, gap_extension1, gap_opening2, gap_extension2; } affine2p_penalties_t;
typedef enum {
    wf_heuristic_none = 0x0,
    wf_heuristic_banded_static = 0x1,
    wf_heuristic_banded_adaptive = 0x2,
    wf_heuristic_wfadaptive = 0x4,
    wf_heuristic_xdrop = 0x10,
    wf_heuristic_zdrop = 0x20,
    wf_heuristic_wfmash = 0x40,
} wf_heuristic_strategy;
typedef struct {
    wf_heuristic_strategy strategy;
    int steps_between_cutoffs, min_k, max_k, min_wavefront_length, max_distance_threshold, xdrop, zdrop;
    int steps_wait, max_sw_score, max_wf_score, max_sw_score_offset, max_sw_score_k;
} wavefront_heuristic_t;
typedef enum {
    wavefront_memory_high = 0,
    wavefront_memory_med = 1,
    wavefront_memory_low = 2,
    wavefront_memory_ultralow = 3,
} wavefront_memory_t;
typedef struct { bool enabled; int resolution_points; int align_level; } wavefront_plot_attr_t;
typedef struct {
    uint64_t total, samples, min, max;
    double m_oldM, m_newM, m_oldS, m_newS;
} profiler_counter_t;
typedef struct {
    struct timespec begin_timer;
    profiler_counter_t time_ns;
    uint64_t accumulated;
} profiler_timer_t;
typedef bool (*wavefront_memory_probe_funct_t)(void *arguments, const uint64_t memory_used,
                                               const uint64_t memory_limit, const int score);
typedef struct {
    int max_alignment_steps;
    int probe_interval_global, probe_interval_compact;
    uint64_t max_partial_compacts, max_memory_compact, max_memory_resident, max_memory_abort;
    uint64_t biwfa_max_memory_abort;
    wavefront_memory_probe_funct_t memory_probe;
    void *memory_probe_arguments;
    int biwfa_leaf_score;
    int verbose;
    bool check_alignment_correct;
    profiler_timer_t timer;
    int max_num_threads, min_offsets_per_thread;
} alignment_system_t;
typedef struct aw_wfa2_mm_allocator mm_allocator_t;  /* only ever a pointer here */
typedef struct {
    distance_metric_t distance_metric;
    alignment_scope_t alignment_scope;
    alignment_form_t alignment_form;
    linear_penalties_t linear_penalties;
    affine_penalties_t affine_penalties;
    affine2p_penalties_t affine2p_penalties;
    wavefront_heuristic_t heuristic;
    wavefront_memory_t memory_mode;
    bool singletrack;
    mm_allocator_t *mm_allocator;
    wavefront_plot_attr_t plot;
    alignment_system_t system;
} wavefront_aligner_attr_t;
#endif /* WAVEFRONT_ATTRIBUTES_H_ */

#ifndef CIGAR_H_
typedef struct {
    char *operations;
    int max_operations;
    int begin_offset, end_offset;
    int score;
    int end_v, end_h;
    bool has_misms;
    uint32_t *cigar_buffer;
    int cigar_length;
} cigar_t;
#endif /* CIGAR_H_ */

#ifndef WF_STATUS_ALG_COMPLETED
#define WF_STATUS_ALG_COMPLETED 0
#define WF_STATUS_OOM (-200)
#define WF_STATUS_UNATTAINABLE (-300)
#endif

/* WFA2-lib's default attributes (wavefront/wavefront_attributes.c:38-106), the values
 * AnchorWave starts from (WfaAlignment.cpp:143) before it sets its own. */
extern const wavefront_aligner_attr_t wavefront_aligner_attr_default_gpu;

/* The members of WFA2-lib's wavefront_align_status_t that callers read (wavefront/wfa.h:
 * status, score, dropped, num_null_steps, memory_used, memory_peak, memory_probe_count,
 * max_num_threads_used); the compute/extend function pointers have no counterpart. */
typedef struct {
    int status;
    int score;
    bool dropped;
    int num_null_steps;
    uint64_t memory_used;         /* device bytes the alignment took from the wavefront pool */
    uint64_t memory_peak;         /* the same (one device pass: the working set at its end) */
    uint64_t memory_probe_count;  /* calls of system.memory_probe made for this alignment */
    int max_num_threads_used;     /* 1 (one warp) */
} wavefront_align_status_gpu_t;

/* The GPU aligner with the members of wavefront_aligner_t that AnchorWave uses. */
typedef struct wavefront_aligner_wfa2_gpu {
    wavefront_align_status_gpu_t align_status;
    cigar_t *cigar;                  /* operations 'M','X','I','D' in [begin_offset, end_offset) */
    alignment_system_t system;       /* the caller may reset memory_probe(_arguments) between calls */
    void *bialigner;                 /* always NULL: BiWFA (ultralow memory) is not provided */
    wavefront_aligner_gpu_t *device; /* the underlying GPU aligner (include/anchorwave_b200.h) */
} wavefront_aligner_wfa2_gpu_t;

/*
 * Replaces wavefront_aligner_new (WFA2-lib wavefront/wfa.h:129-130) for the attributes
 * AnchorWave sets (WfaAlignment.cpp:143-170).  Accepted: distance_metric gap_affine_2p,
 * affine2p_penalties with match 0 and the rest as WFA2-lib takes them (positive), span
 * alignment_end2end without extension, alignment_scope compute_alignment or compute_score,
 * memory_mode high / med / low, singletrack (high memory only, as in WFA2-lib), heuristic
 * wf_heuristic_none, system.max_memory_abort (the device wavefront pool cap; UINT64_MAX =
 * most of the free device memory), system.memory_probe / memory_probe_arguments /
 * probe_interval_global.  Ignored (host threading and diagnostics): max_num_threads,
 * min_offsets_per_thread, verbose, check_alignment_correct, plot, timer, the linear and
 * affine penalty placeholders, max_alignment_steps, the compaction and resident limits,
 * and the BiWFA-only fields.  Anything else (another metric, ends-free or extension
 * alignment, a heuristic, ultralow memory, a caller-owned mm_allocator, match != 0) returns
 * NULL with a message in aw_last_error().
 */
wavefront_aligner_wfa2_gpu_t *wavefront_aligner_new_wfa2_gpu(const wavefront_aligner_attr_t *attributes);

/*
 * Replaces wavefront_align (wfa.h:210-215): pattern = reference, text = query.  Returns
 * the WF status (WF_STATUS_ALG_COMPLETED, WF_STATUS_OOM, WF_STATUS_UNATTAINABLE) and sets
 * align_status and cigar like WFA2-lib (cigar->score = -penalty; an empty CIGAR unless
 * completed).  A device alignment cannot call back into the host while it runs, so the
 * cooperative memory probe is called twice on the host: before the launch with the
 * predicted wavefront bytes and score 0 (admission), and after it with the bytes used and
 * the alignment score; a false return from either reports WF_STATUS_OOM with an empty
 * CIGAR, as when the probe stops WFA2-lib.  Returns AW_E_INVAL for a NULL aligner.
 */
int wavefront_align_wfa2_gpu(wavefront_aligner_wfa2_gpu_t *aligner, const char *pattern, int pattern_length,
                             const char *text, int text_length);

/* Replaces wavefront_aligner_delete. */
void wavefront_aligner_delete_wfa2_gpu(wavefront_aligner_wfa2_gpu_t *aligner);

#ifdef __cplusplus
}
#endif
#endif /* ANCHORWAVE_B200_WFA2_H */
