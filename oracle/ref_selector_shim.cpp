// TEST INFRASTRUCTURE (oracle).  Exposes the compiled selector's sequence pass,
// summarizeSequencePair (src/myImportandFunction/AlignmentAlgorithmSelector.cpp:730-757,
// in an unnamed namespace), to the tests and the CPU leg of bench.py.  The selector's
// source is compiled where it lies, as part of this translation unit; nothing of it is
// copied here.  Nothing in anchorwave_b200/ links or loads it.
#include "AlignmentAlgorithmSelector.cpp"

#include <thread>

namespace {

struct RefSummaryOut {
    uint64_t fingerprint;
    double ambiguous_fraction, normalized_entropy, low_complexity_fraction;
    int64_t count[3];
};

int64_t run_one(const char *query, int64_t qlen, const char *reference, int64_t rlen, const uint64_t *modulos,
                RefSummaryOut *out, int *identical, uint64_t *hash, uint32_t *pos, int64_t cap) {
    using namespace anchorwave;
    const std::string q(query ? query : "", (size_t)qlen), r(reference ? reference : "", (size_t)rlen);
    std::array<uint64_t, kSketchKmerLengths.size()> mod{};
    const uint64_t mx = std::max<uint64_t>(q.size(), r.size());
    for (std::size_t s = 0; s < kSketchKmerLengths.size(); ++s) {
        if (modulos) {
            mod[s] = modulos[s];
        } else {  // as makeAlignmentSelectionPlan derives them
            const uint64_t avail = mx >= kSketchKmerLengths[s] ? mx - kSketchKmerLengths[s] + 1 : 0;
            mod[s] = std::max<uint64_t>(1, avail / kTargetSketchSizes[s]);
        }
    }
    bool ident = false;
    auto sums = summarizeSequencePair(q, r, mod, ident);
    *identical = ident ? 1 : 0;
    int64_t w = 0;
    const SequenceSummary *ss[2] = {&sums.first, &sums.second};
    for (int t = 0; t < 2; ++t) {
        out[t].fingerprint = ss[t]->fingerprint;
        out[t].ambiguous_fraction = ss[t]->ambiguousFraction;
        out[t].normalized_entropy = ss[t]->normalizedEntropy;
        out[t].low_complexity_fraction = ss[t]->lowComplexityFraction;
        for (std::size_t s = 0; s < kSketchKmerLengths.size(); ++s) {
            out[t].count[s] = (int64_t)ss[t]->sketches[s].size();
            for (const SketchEntry &e : ss[t]->sketches[s]) {
                if (hash && w < cap) hash[w] = e.hash, pos[w] = e.position;
                ++w;
            }
        }
    }
    return w;
}

}  // namespace

extern "C" {

int64_t awref_sequence_summary(const char *query, int64_t qlen, const char *reference, int64_t rlen,
                               const uint64_t *modulos, void *out, int *identical, uint64_t *hash, uint32_t *pos,
                               int64_t cap) {
    return run_one(query, qlen, reference, rlen, modulos, (RefSummaryOut *)out, identical, hash, pos, cap);
}

int awref_sizeof_summary(void) { return (int)sizeof(RefSummaryOut); }

// n pairs on nthreads host threads (summaries only, sketches counted, not copied);
// returns the wall seconds.
double awref_sequence_summary_batch(int n, const char *const *query, const int64_t *qlen,
                                    const char *const *reference, const int64_t *rlen, void *out, int *identical,
                                    int nthreads) {
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < n;)
            run_one(query[i], qlen[i], reference[i], rlen[i], nullptr, (RefSummaryOut *)out + 2 * (size_t)i,
                    identical + i, nullptr, nullptr, 0);
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
