// Routing front end of the serving loop (aw_route.h): AnchorWave's selection plan for each
// interval, then the executor's first choice on an idle system.  The selector itself is
// AnchorWave's code, compiled unchanged from its sources by this directory's Makefile; this
// file only calls its public functions in the order the executor does
// (src/myImportandFunction/alignSlidingWindow.cpp:2040-2420).
#include "aw_route.h"

#include <algorithm>
#include <atomic>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "AlignmentAlgorithmSelector.h"

namespace {

using anchorwave::AlignmentCandidate;

const anchorwave::AlgorithmCostEstimate *estimate_of(const anchorwave::AlignmentSelectionPlan &p,
                                                     AlignmentCandidate c) {
    for (const auto &e : p.estimates)
        if (e.candidate == c) return &e;
    return nullptr;
}

bool is_wfa(AlignmentCandidate c) {
    return c == AlignmentCandidate::SingletrackWfa || c == AlignmentCandidate::StandardWfa ||
           c == AlignmentCandidate::MediumWfa || c == AlignmentCandidate::LowWfa;
}

aw_serve_route_t route_of(AlignmentCandidate c, const anchorwave::AlignmentSelectionPlan &p) {
    aw_serve_route_t r;
    r.band = -1, r.band_max = -1, r.window = 0;
    const anchorwave::AlgorithmCostEstimate *e = estimate_of(p, c);
    r.predicted_bytes = e ? (int64_t)std::min<uint64_t>(e->memoryBytes, (uint64_t)INT64_MAX) : 0;
    switch (c) {
    case AlignmentCandidate::SingletrackWfa: r.method = AW_ROUTE_WFA_SINGLETRACK; break;
    case AlignmentCandidate::StandardWfa: r.method = AW_ROUTE_WFA; break;
    case AlignmentCandidate::MediumWfa: r.method = AW_ROUTE_WFA_MEDIUM; break;
    case AlignmentCandidate::LowWfa: r.method = AW_ROUTE_WFA_LOW; break;
    case AlignmentCandidate::Ksw2Singletrack: r.method = AW_ROUTE_KSW2_SINGLETRACK; break;
    case AlignmentCandidate::Ksw2Full: r.method = AW_ROUTE_KSW2; break;
    case AlignmentCandidate::Ksw2ScoreCertified:
        r.method = AW_ROUTE_KSW2_CERTIFIED;
        r.band = (int)std::min<int64_t>(p.ksw2CertifiedInitialBandWidth, std::numeric_limits<int>::max());
        r.band_max = (int)std::min<int64_t>(p.ksw2CertifiedMaximumBandWidth, std::numeric_limits<int>::max());
        break;
    case AlignmentCandidate::Ksw2Banded:
        r.method = AW_ROUTE_KSW2;
        r.band = (int)std::min<int64_t>(p.ksw2BandWidth, std::numeric_limits<int>::max());
        break;
    case AlignmentCandidate::SlidingWindow:
    default:
        r.method = AW_ROUTE_SLIDING_WINDOW;
        r.window = p.slidingWindowWidth;
        break;
    }
    return r;
}

aw_route_choice_t choose(const std::string &q, const std::string &d, int64_t window, int mis, int o1, int e1,
                         int o2, int e2) {
    const anchorwave::AlignmentSelectionPlan p =
            anchorwave::makeAlignmentSelectionPlan(q, d, window, mis, o1, e1, o2, e2);
    std::vector<AlignmentCandidate> ranked;
    for (AlignmentCandidate c : p.exactCandidates)
        if (estimate_of(p, c)) ranked.push_back(c);
    // the executor's pruning (alignSlidingWindow.cpp:2180-2245)
    const bool has_full = std::count(ranked.begin(), ranked.end(), AlignmentCandidate::Ksw2Full) > 0;
    const bool has_st = std::count(ranked.begin(), ranked.end(), AlignmentCandidate::Ksw2Singletrack) > 0;
    if (has_full && has_st &&
        anchorwave::exactCandidateEpsilonDominates(*estimate_of(p, AlignmentCandidate::Ksw2Full),
                                                   *estimate_of(p, AlignmentCandidate::Ksw2Singletrack), 0.002))
        ranked.erase(std::remove(ranked.begin(), ranked.end(), AlignmentCandidate::Ksw2Singletrack), ranked.end());
    const bool full_now = std::count(ranked.begin(), ranked.end(), AlignmentCandidate::Ksw2Full) > 0;
    if (anchorwave::deferScoreCertifiedKsw2BehindFullKsw2(false, full_now))
        ranked.erase(std::remove(ranked.begin(), ranked.end(), AlignmentCandidate::Ksw2ScoreCertified), ranked.end());
    const bool independent = std::any_of(ranked.begin(), ranked.end(), [](AlignmentCandidate c) {
        return anchorwave::isIndependentExactAfterSingletrackMemoryFailure(c);
    });
    if (independent && anchorwave::preferIndependentKsw2ForAmbiguousWfaProfile(p.profile))
        ranked.erase(std::remove_if(ranked.begin(), ranked.end(), is_wfa), ranked.end());
    aw_route_choice_t out;
    if (!ranked.empty()) {
        // expected completion over the failure chain (:2313-2340), no wait, one active task
        std::vector<anchorwave::ExactAttemptSystemCost> attempts;
        for (AlignmentCandidate c : ranked) {
            const anchorwave::AlgorithmCostEstimate eff =
                    anchorwave::calibratedAlignmentCostEstimate(*estimate_of(p, c), 1, 1);
            attempts.push_back(anchorwave::ExactAttemptSystemCost{c, anchorwave::alignmentRiskAdjustedMinutes(eff),
                                                                  eff.successProbability});
        }
        size_t best = 0;
        double best_cost = std::numeric_limits<double>::infinity();
        for (size_t i = 0; i < ranked.size(); ++i) {
            const double cost = anchorwave::exactAttemptExpectedSystemMinutes(attempts, i);
            if (cost < best_cost) best = i, best_cost = cost;
        }
        out.route = route_of(ranked[best], p);
        out.candidate = (int)ranked[best];
        out.tier = 1;
    } else {
        const AlignmentCandidate c = p.approximateDecision.selected;
        out.route = route_of(c, p);
        out.candidate = (int)c;
        out.tier = 2;
    }
    return out;
}

}  // namespace

extern "C" int aw_route_intervals(int n, const char *const *query, const int64_t *qlen,
                                  const char *const *reference, const int64_t *rlen, int64_t window_width,
                                  int32_t mis, int32_t o1, int32_t e1, int32_t o2, int32_t e2, int nthreads,
                                  aw_route_choice_t *out) {
    if (n < 0 || (n > 0 && (!query || !qlen || !reference || !rlen || !out))) return -1;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < n;) {
            const std::string q(query[i] ? query[i] : "", (size_t)qlen[i]);
            const std::string d(reference[i] ? reference[i] : "", (size_t)rlen[i]);
            out[i] = choose(q, d, window_width, mis, o1, e1, o2, e2);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < std::max(1, nthreads); ++t) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
    return 0;
}
