/*
 * aw_route.h -- routing front end of the serving loop (libaw_route.so).
 *
 * AnchorWave picks each interval's engine with its exact-tier / fallback-tier selector
 * (makeAlignmentSelectionPlan, src/myImportandFunction/AlignmentAlgorithmSelector.cpp:1711)
 * and its executor's ranking (alignSlidingWindow.cpp:2040-2420).  This library links that
 * selector, compiled unchanged from AnchorWave's sources, and returns for every interval the
 * route of include/anchorwave_b200.h (engine and parameters) that the executor starts
 * first on an idle system: every engine's memory ready, no wait and one active task, so the
 * memory opportunity cost is zero and the choice is the exact candidate with the smallest
 * expected completion over its failure chain (exactAttemptExpectedSystemMinutes of the
 * calibrated, risk-adjusted estimates), after the executor's pruning rules; with no exact
 * candidate, the approximate tier's predicted winner (banded KSW2 or sliding window).
 */
#ifndef AW_ROUTE_H
#define AW_ROUTE_H

#include <stdint.h>

#include "../../include/anchorwave_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    aw_serve_route_t route;   /* route.predicted_bytes: the plan's memoryBytes of the candidate */
    int candidate;  /* anchorwave::AlignmentCandidate (AlignmentAlgorithmSelector.h:10-20) */
    int tier;       /* 1 exact, 2 approximate */
} aw_route_choice_t;

/* Routes n intervals (ASCII) on nthreads host threads with the selector's inputs: the -w
 * window width and AnchorWave's penalties (negative).  Returns 0, or -1 on bad arguments. */
int aw_route_intervals(int n, const char *const *query, const int64_t *qlen, const char *const *reference,
                       const int64_t *rlen, int64_t window_width, int32_t mismatching_penalty, int32_t open1,
                       int32_t extend1, int32_t open2, int32_t extend2, int nthreads, aw_route_choice_t *out);

#ifdef __cplusplus
}
#endif
#endif /* AW_ROUTE_H */
