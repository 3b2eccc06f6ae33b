// WFA2-lib-typed front end of the GPU WFA aligner (include/anchorwave_b200_wfa2.h):
// takes the wavefront_aligner_attr_t that AnchorWave builds
// (src/myImportandFunction/WfaAlignment.cpp:143-170), checks that it asks for what the
// device aligner computes, and returns an aligner whose align_status / cigar / system /
// bialigner members are the ones AnchorWave reads after wavefront_align
// (WfaAlignment.cpp:343-356).  Host code only; the alignment itself is
// wavefront_align_gpu (wfa_api.cu).
#include "aw_internal.h"
#include "../../include/anchorwave_b200_wfa2.h"

#include <climits>
#include <string>
#include <cstdlib>
#include <cstring>
#include <new>

// WFA2-lib's defaults, wavefront/wavefront_attributes.c:38-106 (heuristic wfadaptive,
// metric gap_affine, penalties 0/4/6/2/24/1, high memory, unlimited memory).
extern "C" const wavefront_aligner_attr_t wavefront_aligner_attr_default_gpu = [] {
    wavefront_aligner_attr_t a;
    memset(&a, 0, sizeof(a));
    a.distance_metric = gap_affine;
    a.alignment_scope = compute_alignment;
    a.alignment_form.span = alignment_end2end;
    a.alignment_form.extension = false;
    a.linear_penalties = {0, 4, 2};
    a.affine_penalties = {0, 4, 6, 2};
    a.affine2p_penalties = {0, 4, 6, 2, 24, 1};
    a.heuristic.strategy = wf_heuristic_wfadaptive;
    a.heuristic.min_wavefront_length = 10;
    a.heuristic.max_distance_threshold = 50;
    a.heuristic.steps_between_cutoffs = 1;
    a.memory_mode = wavefront_memory_high;
    a.singletrack = false;
    a.mm_allocator = nullptr;
    a.plot.enabled = false, a.plot.resolution_points = 2000, a.plot.align_level = 0;
    a.system.max_alignment_steps = INT_MAX;
    a.system.probe_interval_global = 3000;
    a.system.probe_interval_compact = 6000;
    a.system.max_memory_compact = (uint64_t)-1;
    a.system.max_memory_resident = (uint64_t)-1;
    a.system.max_memory_abort = UINT64_MAX;
    a.system.biwfa_max_memory_abort = UINT64_MAX;
    a.system.memory_probe = nullptr;
    a.system.memory_probe_arguments = nullptr;
    a.system.biwfa_leaf_score = 250;
    a.system.verbose = 0;
    a.system.check_alignment_correct = false;
    a.system.max_num_threads = 1;
    a.system.min_offsets_per_thread = 500;
    return a;
}();

namespace {

// Penalties as WFA2-lib normalises them (wavefront/wavefront_penalties.c:141-150 takes
// the absolute values of negative gap and mismatch penalties).
int pos(int p) { return p < 0 ? -p : p; }

// Wavefront bytes a pair is predicted to take (admission probe): the retained offsets
// grow with the square of the alignment score, bounded here by a length-based proxy
// (five components of 4-byte offsets in high memory, M only in Singletrack, a ring plus
// packed-CIGAR blocks in the piggyback modes).
uint64_t predicted_bytes(int plen, int tlen, int memory_mode, bool singletrack) {
    const uint64_t L = (uint64_t)plen + (uint64_t)tlen;
    const uint64_t div = memory_mode > 0 ? 128 : singletrack ? 64 : 16;
    return 64 * L + L * L / div;
}

struct AlignerBox {
    wavefront_aligner_wfa2_gpu_t pub;
    cigar_t cigar;
    char *ops = nullptr;
    int ops_cap = 0;
    bool score_only = false;
    int memory_mode = 0;
    bool singletrack = false;
};

}  // namespace

using namespace aw;

extern "C" {

wavefront_aligner_wfa2_gpu_t *wavefront_aligner_new_wfa2_gpu(const wavefront_aligner_attr_t *a) {
    if (!a) {
        set_error("wavefront_aligner_new_wfa2_gpu: attributes required");
        return nullptr;
    }
    const char *why = nullptr;
    if (a->distance_metric != gap_affine_2p) why = "distance_metric must be gap_affine_2p";
    else if (a->affine2p_penalties.match != 0) why = "affine2p_penalties.match must be 0";
    else if (a->alignment_form.span != alignment_end2end || a->alignment_form.extension)
        why = "only end-to-end alignment (alignment_end2end, no extension) is provided";
    else if (a->alignment_scope != compute_alignment && a->alignment_scope != compute_score)
        why = "alignment_scope must be compute_alignment or compute_score";
    else if (a->heuristic.strategy != wf_heuristic_none) why = "heuristic.strategy must be wf_heuristic_none";
    else if (a->memory_mode != wavefront_memory_high && a->memory_mode != wavefront_memory_med &&
             a->memory_mode != wavefront_memory_low)
        why = "memory_mode must be high, med or low (ultralow / BiWFA is not provided)";
    else if (a->mm_allocator) why = "a caller-owned mm_allocator is not supported (device memory is pooled)";
    if (why) {
        set_error((std::string("wavefront_aligner_new_wfa2_gpu: ") + why).c_str());
        return nullptr;
    }
    wavefront_gpu_attr_t g;
    g.mismatch = pos(a->affine2p_penalties.mismatch);
    g.gap_opening1 = pos(a->affine2p_penalties.gap_opening1);
    g.gap_extension1 = pos(a->affine2p_penalties.gap_extension1);
    g.gap_opening2 = pos(a->affine2p_penalties.gap_opening2);
    g.gap_extension2 = pos(a->affine2p_penalties.gap_extension2);
    // wavefront/wavefront_aligner.c:251-260: Singletrack only in high memory
    g.singletrack = (a->singletrack && a->memory_mode == wavefront_memory_high) ? 1 : 0;
    g.memory_mode = (int)a->memory_mode;
    g.max_memory_abort = (a->system.max_memory_abort == UINT64_MAX || a->system.max_memory_abort > (uint64_t)INT64_MAX)
                             ? 0
                             : (int64_t)a->system.max_memory_abort;
    wavefront_aligner_gpu_t *dev = wavefront_aligner_new_gpu(&g);
    if (!dev) return nullptr;  // the message is already set
    AlignerBox *box = new (std::nothrow) AlignerBox();
    if (!box) {
        wavefront_aligner_delete_gpu(dev);
        set_error("wavefront_aligner_new_wfa2_gpu: out of host memory");
        return nullptr;
    }
    memset(&box->pub, 0, sizeof(box->pub));
    memset(&box->cigar, 0, sizeof(box->cigar));
    box->pub.cigar = &box->cigar;
    box->pub.system = a->system;
    box->pub.bialigner = nullptr;
    box->pub.device = dev;
    box->pub.align_status.max_num_threads_used = 1;
    box->score_only = a->alignment_scope == compute_score;
    box->memory_mode = (int)a->memory_mode;
    box->singletrack = g.singletrack != 0;
    return &box->pub;
}

int wavefront_align_wfa2_gpu(wavefront_aligner_wfa2_gpu_t *al, const char *pattern, int pattern_length,
                             const char *text, int text_length) {
    if (!al) return AW_E_INVAL;
    AlignerBox *box = reinterpret_cast<AlignerBox *>(al);
    wavefront_align_status_gpu_t &S = al->align_status;
    cigar_t &cg = box->cigar;
    S.status = WF_STATUS_OOM, S.score = 0, S.dropped = false, S.num_null_steps = 0;
    S.memory_used = 0, S.memory_peak = 0, S.memory_probe_count = 0;
    cg.begin_offset = cg.end_offset = 0, cg.score = 0, cg.end_v = cg.end_h = 0;
    cg.has_misms = false, cg.cigar_buffer = nullptr, cg.cigar_length = 0;
    const alignment_system_t &sys = al->system;
    const uint64_t limit = sys.max_memory_abort;
    if (sys.memory_probe) {
        ++S.memory_probe_count;
        const uint64_t pred = predicted_bytes(pattern_length, text_length, box->memory_mode, box->singletrack);
        if (!sys.memory_probe(sys.memory_probe_arguments, pred, limit, 0)) return S.status = WF_STATUS_OOM;
    }
    const int st = wavefront_align_gpu(al->device, pattern, pattern_length, text, text_length);
    if (st != WF_STATUS_ALG_COMPLETED && st != WF_STATUS_OOM && st != WF_STATUS_UNATTAINABLE) {
        // a CUDA or argument failure of the device aligner: reported as the abort status
        S.status = WF_STATUS_OOM;
        return S.status;
    }
    int64_t used = 0;
    wavefront_gpu_memory(al->device, &used, nullptr);
    S.memory_used = S.memory_peak = (uint64_t)used;
    S.status = st;
    if (st != WF_STATUS_ALG_COMPLETED) return st;
    const char *ops = nullptr;
    int nops = 0, score = 0;
    wavefront_gpu_cigar(al->device, &ops, &nops, &score);
    if (sys.memory_probe) {
        ++S.memory_probe_count;
        if (!sys.memory_probe(sys.memory_probe_arguments, S.memory_used, limit, -score))
            return S.status = WF_STATUS_OOM;
    }
    // align_status.score is the wavefront score (the penalty, wavefront_unialign.c:105-151);
    // cigar->score the classic score, -penalty with match 0 (wavefront_unialign.c:247)
    S.score = -score;
    cg.score = score;
    cg.end_v = pattern_length, cg.end_h = text_length;
    if (!box->score_only) {
        if (nops + 1 > box->ops_cap) {
            char *p = (char *)realloc(box->ops, (size_t)nops + 1);
            if (!p) {
                set_error("wavefront_align_wfa2_gpu: out of host memory");
                return S.status = WF_STATUS_OOM;
            }
            box->ops = p, box->ops_cap = nops + 1;
        }
        memcpy(box->ops, ops, (size_t)nops);
        box->ops[nops] = 0;
        cg.operations = box->ops, cg.max_operations = box->ops_cap;
        cg.begin_offset = 0, cg.end_offset = nops;
    }
    return st;
}

void wavefront_aligner_delete_wfa2_gpu(wavefront_aligner_wfa2_gpu_t *al) {
    if (!al) return;
    AlignerBox *box = reinterpret_cast<AlignerBox *>(al);
    wavefront_aligner_delete_gpu(al->device);
    free(box->ops);
    delete box;
}

}  // extern "C"
