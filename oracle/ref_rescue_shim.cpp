// TEST INFRASTRUCTURE (oracle).  Exposes AnchorWave's own rescue procedures and its KSW2
// row decoding from the compiled reference to the tests:
//   * alignScoreCertifiedKsw2 (src/myImportandFunction/alignSlidingWindow.cpp:1197-1400);
//   * the semiglobal sliding-window alignment alignSlidingWindow (:457-590);
//   * alignSlidingWindow_minimap2 (the banded KSW2 call, decoding and re-scoring);
//   * minimap2AlignmentWithArena (:241-332: one global KSW2 call and the CIGAR -> gapped rows
//     decoding of :307-324).
// The reference source is compiled where it lies, as part of this translation unit (so
// that its file-scope functions are reachable); nothing of it is copied here.  Nothing in
// anchorwave_b200/ links or loads it.
#include "alignSlidingWindow.cpp"

#include <cstring>

namespace {

int64_t put_rows(const std::string &q, const std::string &d, char *out_q, char *out_d, int64_t cap) {
    const int64_t n = (int64_t)q.size();
    if ((int64_t)d.size() != n) return -1;
    if (out_q && out_d && n <= cap) {
        memcpy(out_q, q.data(), (size_t)n);
        memcpy(out_d, d.data(), (size_t)n);
    }
    return n;
}

}  // namespace

extern "C" {

// alignScoreCertifiedKsw2 with no selection plan and no deadline.  Penalties as AnchorWave
// passes them (negative).  Returns the status (Ksw2CertifiedStatus as int); the rows go to
// out_q/out_d (*out_len characters, -1 if beyond cap), the best-effort rows to be_q/be_d.
int awref_score_certified(const char *q, int64_t ql, const char *d, int64_t dl, int64_t initial_band,
                          int64_t maximum_band, int mis, int o1, int e1, int o2, int e2, int64_t *score,
                          int64_t *optimal, int64_t *final_band, int64_t *attempts, char *out_q, char *out_d,
                          int64_t cap, int64_t *out_len, char *be_q, char *be_d, int64_t *be_len) {
    const std::string dq(q, (size_t)ql), dd(d, (size_t)dl);
    std::string aq, ad;
    const int32_t m = mis, go1 = o1, ge1 = e1, go2 = o2, ge2 = e2;
    const anchorwave::Ksw2CertifiedResult r =
            alignScoreCertifiedKsw2(dq, dd, aq, ad, initial_band, maximum_band, 0.0, m, go1, ge1, go2, ge2);
    *score = r.score;
    *optimal = r.optimalScore;
    *final_band = r.finalBandWidth;
    *attempts = (int64_t)r.tracebackAttempts;
    *out_len = put_rows(aq, ad, out_q, out_d, cap);
    *be_len = put_rows(r.bestEffortQueryAlignment, r.bestEffortReferenceAlignment, be_q, be_d, cap);
    return (int)r.status;
}

// alignSlidingWindow (the semiglobal-window form, alignSlidingWindow.cpp:457-590): returns the
// re-scored score; rows as above.
int64_t awref_sliding_window(const char *q, int64_t ql, const char *d, int64_t dl, int64_t window, int match,
                             int mis, int o1, int e1, int o2, int e2, char *out_q, char *out_d, int64_t cap,
                             int64_t *out_len) {
    const std::string dq(q, (size_t)ql), dd(d, (size_t)dl);
    std::string aq, ad;
    const int32_t mt = match, m = mis, go1 = o1, ge1 = e1, go2 = o2, ge2 = e2;
    const int64_t s = alignSlidingWindow(dq, dd, ql, dl, aq, ad, window, mt, m, go1, ge1, go2, ge2);
    *out_len = put_rows(aq, ad, out_q, out_d, cap);
    return s;
}

// minimap2AlignmentWithArena: one global ksw_extd2 call of the native ISA and the CIGAR
// decoded into gapped rows (:307-324).  Returns ez.score.
int64_t awref_minimap2_rows(const char *q, int64_t ql, const char *d, int64_t dl, int mis, int o1, int e1, int o2,
                            int e2, char *out_q, char *out_d, int64_t cap, int64_t *out_len) {
    const std::string dq(q, (size_t)ql), dd(d, (size_t)dl);
    std::string aq, ad;
    const int32_t mt = 0;
    const int64_t s = minimap2AlignmentWithArena(nullptr, dq, dd, aq, ad, mt, mis, o1, e1, o2, e2);
    *out_len = put_rows(aq, ad, out_q, out_d, cap);
    return s;
}

// alignSlidingWindow_minimap2 at band width `band` (-1: full): decoded rows and their
// two-piece affine re-score.
int64_t awref_banded_rows(const char *q, int64_t ql, const char *d, int64_t dl, int64_t band, int mis, int o1, int e1,
                          int o2, int e2, char *out_q, char *out_d, int64_t cap, int64_t *out_len) {
    const std::string dq(q, (size_t)ql), dd(d, (size_t)dl);
    std::string aq, ad;
    const int32_t m = mis, go1 = o1, ge1 = e1, go2 = o2, ge2 = e2;
    const int64_t s = alignSlidingWindow_minimap2(dq, dd, ql, dl, aq, ad, band, m, go1, ge1, go2, ge2);
    *out_len = put_rows(aq, ad, out_q, out_d, cap);
    return s;
}

}  // extern "C"
