// Exact anti-diagonal KSW2 kernel (all flags, banded, Singletrack): host entry.
#pragma once
#include "aw_internal.h"
#include <vector>

namespace aw {

// SIMD width (bytes) of the reference kernel whose padding semantics the exact
// kernel reproduces: 64 = ksw_extd2_avx512, 32 = ksw_extd2_avx2, 16 = ksw_extd2_sse.
int exact_block();
void set_exact_block(int b);
// Cooperative-stop emulation (minimap2/ksw2_progress.c:30-38): stop at the first
// probed anti-diagonal r (r % interval == 0) with r >= stop_at; stop_at < 0 disables.
// Per calling thread.
void set_exact_stop(int interval, int stop_at);
bool exact_stop_enabled();

int run_exact_ksw(size_t n_exact, const int32_t *d_ids, const uint8_t *d_q, const uint8_t *d_t,
                  const KswPair *d_pairs, const std::vector<KswPair> &h_pairs,
                  const std::vector<int32_t> &ids, const std::vector<int> &w, int m,
                  const int8_t *mat, const KswScore &S, int zdrop, int end_bonus, int flag,
                  KswOut *d_out, uint32_t *d_cig, DevBuf &ws, cudaStream_t st, int *launches,
                  const unsigned long long *deadline = nullptr);

}  // namespace aw
