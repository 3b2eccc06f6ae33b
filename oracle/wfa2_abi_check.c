/* TEST INFRASTRUCTURE.  A WFA2-lib caller, written as AnchorWave's WFA adapter is
 * (src/myImportandFunction/WfaAlignment.cpp:143-170, :343-356): it includes WFA2-lib's own
 * wavefront/wfa.h, builds wavefront_aligner_attr_t from WFA2-lib's
 * wavefront_aligner_attr_default, and aligns every pair twice with those same attributes:
 * with the compiled WFA2-lib (wavefront_aligner_new / wavefront_align) and through the GPU
 * library's WFA2-typed entries (include/anchorwave_b200_wfa2.h).  It compares status,
 * align_status.score, cigar->score and the operations [begin_offset, end_offset), and counts
 * the memory-probe calls.  Built by oracle/Makefile (it needs the reference tree's headers),
 * run by tests/test_wfa2_boundary.py on a GPU.
 *
 * usage: wfa2_abi_check <pairs file: pattern TAB text per line> <memory_mode 0|1|2> <singletrack 0|1>
 * prints "pairs N identical M probe_calls P" and exits 0 when every pair agrees. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wavefront/wfa.h"
#include "anchorwave_b200_wfa2.h"

static int g_probe_calls = 0;

static bool count_probe(void *arguments, const uint64_t memory_used, const uint64_t memory_limit, const int score) {
    (void)arguments, (void)memory_used, (void)memory_limit, (void)score;
    ++g_probe_calls;
    return true;
}

static wavefront_aligner_attr_t anchorwave_attributes(int memory_mode, int singletrack) {
    wavefront_aligner_attr_t attributes = wavefront_aligner_attr_default;
    attributes.distance_metric = gap_affine_2p;
    attributes.affine2p_penalties.match = 0;
    attributes.affine2p_penalties.mismatch = 4;
    attributes.affine2p_penalties.gap_opening1 = 4;
    attributes.affine2p_penalties.gap_extension1 = 2;
    attributes.affine2p_penalties.gap_opening2 = 24;
    attributes.affine2p_penalties.gap_extension2 = 1;
    attributes.alignment_form.span = alignment_end2end;
    attributes.alignment_scope = compute_alignment;
    attributes.memory_mode = (wavefront_memory_t)memory_mode;
    attributes.singletrack = singletrack != 0;
    attributes.heuristic.strategy = wf_heuristic_none;
    attributes.system.max_memory_abort = UINT64_MAX;
    attributes.system.probe_interval_global = 3000;
    attributes.system.memory_probe = count_probe;
    attributes.system.memory_probe_arguments = NULL;
    attributes.system.verbose = 0;
    attributes.system.max_num_threads = 1;
    return attributes;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s pairs.tsv memory_mode singletrack\n", argv[0]);
        return 2;
    }
    const int mode = atoi(argv[2]), st = atoi(argv[3]);
    FILE *f = fopen(argv[1], "r");
    if (!f) return 2;
    wavefront_aligner_attr_t attributes = anchorwave_attributes(mode, st);
    wavefront_aligner_t *ref = wavefront_aligner_new(&attributes);
    wavefront_aligner_wfa2_gpu_t *gpu = wavefront_aligner_new_wfa2_gpu(&attributes);
    if (!ref || !gpu) {
        fprintf(stderr, "aligner creation failed: %s\n", aw_last_error());
        return 3;
    }
    if (gpu->bialigner != NULL) return 4;
    size_t cap = 0;
    char *line = NULL;
    int pairs = 0, identical = 0, gpu_probe_calls = 0;
    while (getline(&line, &cap, f) > 0) {
        char *tab = strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        char *pat = line, *txt = tab + 1;
        size_t tl = strlen(txt);
        while (tl && (txt[tl - 1] == '\n' || txt[tl - 1] == '\r')) txt[--tl] = 0;
        const int pl = (int)strlen(pat);
        g_probe_calls = 0;
        const int rs = wavefront_align(ref, pat, pl, txt, (int)tl);
        g_probe_calls = 0;
        const int gs = wavefront_align_wfa2_gpu(gpu, pat, pl, txt, (int)tl);
        gpu_probe_calls += g_probe_calls;
        int same = rs == gs && gpu->align_status.status == gs && (int)gpu->align_status.memory_probe_count == g_probe_calls;
        if (same && rs == WF_STATUS_ALG_COMPLETED) {
            const cigar_t *a = ref->cigar, *b = gpu->cigar;
            const int na = a->end_offset - a->begin_offset, nb = b->end_offset - b->begin_offset;
            same = a->score == b->score && ref->align_status.score == gpu->align_status.score && na == nb &&
                   memcmp(a->operations + a->begin_offset, b->operations + b->begin_offset, (size_t)na) == 0 &&
                   gpu->align_status.memory_used > 0 && gpu->align_status.memory_peak >= gpu->align_status.memory_used;
        }
        if (!same)
            fprintf(stderr, "pair %d (%d x %zu) differs: status %d / %d, score %d / %d\n", pairs, pl, tl, rs, gs,
                    ref->cigar->score, gpu->cigar->score);
        ++pairs;
        identical += same;
    }
    free(line);
    fclose(f);
    wavefront_aligner_delete(ref);
    wavefront_aligner_delete_wfa2_gpu(gpu);
    printf("pairs %d identical %d probe_calls %d\n", pairs, identical, gpu_probe_calls);
    return identical == pairs && pairs > 0 ? 0 : 1;
}
