/* TEST INFRASTRUCTURE.  Prints the size and member offsets of wavefront_aligner_attr_t
 * and cigar_t.  Compiled twice by tests/test_wfa2_boundary.py: with -DAW_WITH_WFA2 the
 * types come from WFA2-lib's own headers in the reference tree (wavefront/wfa.h), without
 * it from include/anchorwave_b200_wfa2.h; the two outputs must be identical for the GPU
 * entries to accept the struct a WFA2-lib caller builds. */
#include <stddef.h>
#include <stdio.h>
#ifdef AW_WITH_WFA2
#include "wavefront/wfa.h"
#endif
#include "anchorwave_b200_wfa2.h"

#define P(T, m) printf("%s.%s %zu\n", #T, #m, offsetof(T, m))

int main(void) {
    printf("sizeof(wavefront_aligner_attr_t) %zu\n", sizeof(wavefront_aligner_attr_t));
    P(wavefront_aligner_attr_t, distance_metric);
    P(wavefront_aligner_attr_t, alignment_scope);
    P(wavefront_aligner_attr_t, alignment_form);
    P(wavefront_aligner_attr_t, alignment_form.extension);
    P(wavefront_aligner_attr_t, alignment_form.text_end_free);
    P(wavefront_aligner_attr_t, linear_penalties);
    P(wavefront_aligner_attr_t, affine_penalties);
    P(wavefront_aligner_attr_t, affine2p_penalties);
    P(wavefront_aligner_attr_t, affine2p_penalties.mismatch);
    P(wavefront_aligner_attr_t, affine2p_penalties.gap_extension2);
    P(wavefront_aligner_attr_t, heuristic);
    P(wavefront_aligner_attr_t, heuristic.max_sw_score_k);
    P(wavefront_aligner_attr_t, memory_mode);
    P(wavefront_aligner_attr_t, singletrack);
    P(wavefront_aligner_attr_t, mm_allocator);
    P(wavefront_aligner_attr_t, plot);
    P(wavefront_aligner_attr_t, system);
    P(wavefront_aligner_attr_t, system.probe_interval_global);
    P(wavefront_aligner_attr_t, system.max_memory_abort);
    P(wavefront_aligner_attr_t, system.biwfa_max_memory_abort);
    P(wavefront_aligner_attr_t, system.memory_probe);
    P(wavefront_aligner_attr_t, system.memory_probe_arguments);
    P(wavefront_aligner_attr_t, system.biwfa_leaf_score);
    P(wavefront_aligner_attr_t, system.verbose);
    P(wavefront_aligner_attr_t, system.check_alignment_correct);
    P(wavefront_aligner_attr_t, system.timer);
    P(wavefront_aligner_attr_t, system.max_num_threads);
    P(wavefront_aligner_attr_t, system.min_offsets_per_thread);
    printf("sizeof(cigar_t) %zu\n", sizeof(cigar_t));
    P(cigar_t, operations);
    P(cigar_t, max_operations);
    P(cigar_t, begin_offset);
    P(cigar_t, end_offset);
    P(cigar_t, score);
    P(cigar_t, end_v);
    P(cigar_t, end_h);
    P(cigar_t, has_misms);
    P(cigar_t, cigar_buffer);
    P(cigar_t, cigar_length);
    printf("enum gap_affine_2p %d wavefront_memory_low %d wf_heuristic_none %d compute_alignment %d "
           "alignment_end2end %d\n", (int)gap_affine_2p, (int)wavefront_memory_low, (int)wf_heuristic_none,
           (int)compute_alignment, (int)alignment_end2end);
    return 0;
}
