// Banded strip kernel for KSW2 extd2 (w >= 0, and the Singletrack traceback at any w):
// host-side planning and launch interface.
#pragma once
#include "aw_internal.h"
#include <vector>

namespace aw {

// One pair as the banded kernel sees it (device layout).
struct BandPairDev {
    int64_t qoff, toff;     // code offsets in the sequence arenas
    int64_t cig_off;        // word offset of the CIGAR slot (capacity qlen+tlen+2)
    int32_t qlen, tlen, w;  // w >= 0 (a full-width band is w = max(qlen, tlen))
    int32_t rb;             // first anti-diagonal the reference does not compute (band break), else qlen+tlen-1
    int32_t strip0;         // index of this pair's first strip descriptor
    int32_t nstrip;
    int32_t idx;            // pair index in the batch (KswOut / KswPair arrays)
    int32_t ckpt;           // 1: traceback too large for the budget; recomputed strip group by group
};

// One 256-column strip: the rows it sweeps and where its traceback and its right-edge
// column (read by the next strip) live.
struct BandStripDev {
    int64_t tb_off;   // bytes into the traceback arena (CIGAR modes)
    int64_t bnd_off;  // uint2 entries into the boundary arena
    int32_t jstart;   // first row swept (may be negative: score-fill rows above the matrix)
    int32_t jlo;      // first stored row, max(0, jstart)
    int32_t jend;     // last row swept (< jlo: empty strip)
    int32_t pad;
};

// Per-pair end tracking merged across strips: (value, position) packed so that an
// unsigned max keeps the largest value and, among equal values, the later position.
struct BandRes {
    unsigned long long mqe_key, mte_key;
    int32_t score, has_score;
    int32_t stopped;  // a strip of the pair saw the calling thread's deadline pass
    int32_t pad;
};

struct BandWave {
    int pair0, npair;    // slots [pair0, pair0 + npair) of the pair table
    int unit0, nunit;    // units [unit0, unit0 + nunit) of the unit table
    int strip0, nstrip;  // strip descriptors used by this wave
    int64_t tb_bytes, bnd_entries;
    int round0, nround;  // recompute rounds of this wave's recomputed pairs, in walk order
};

// Walk state of a pair whose traceback is recomputed group by group (see band_plan_build).
struct BandWalkState {
    int32_t i, j, state;   // ksw_backtrack position and state
    int32_t n, op, len;    // CIGAR runs written, the open run
    int32_t done, pad;     // 1: nothing (left) to walk
};

// A group of consecutive strips of one recomputed pair (device layout): its strips run again
// with their traceback stored, then the pair's walk continues through them.  The walk visits
// a pair's groups from the last to the first.
struct BandGroupDev {
    int32_t slot;             // pair slot
    int32_t s_first, s_end;   // strip descriptors [s_first, s_end) (global indices)
    int32_t left;             // the strip on the group's left (its stored column is the input), or -1
    int32_t col_lo;           // first target column of the group
    int32_t last;             // 1: the pair's first group (the walk ends here)
    int32_t pad0, pad1;
};

// One recompute round of a wave: one group of every recomputed pair that still has one, run
// together (their strips in one launch, their walks in another); the groups of a round share
// the traceback arena, each at its own offset.
struct BandRound {
    int group0, ngroup;  // groups [group0, group0 + ngroup) of the group table
    int unit0, nunit;    // their strips, in estimated start order
    int nstrip;          // strips to reset
    int64_t tb_bytes;
};

struct BandPlan {
    std::vector<BandPairDev> pairs;
    std::vector<BandGroupDev> groups;
    std::vector<BandRound> rounds;
    std::vector<BandStripDev> strips;
    std::vector<int2> units;  // (pair slot, strip) in processing order
    std::vector<BandWave> waves;
    int64_t tb_cap = 0, bnd_cap = 0, tb_total = 0, cells = 0;
    int block = 64;
    int nc = 8;  // target columns per lane: strips of 32*nc columns
};

// Geometry of the reference's band (ksw2_extd2_sse.c:147-154): the first anti-diagonal
// whose band is empty (the reference stops there with zdropped = 1), or qlen+tlen-1.
int band_break(int qlen, int tlen, int w);

// Sum over anti-diagonals of the in-band cell count en0-st0+1 up to the band break.
int64_t band_cells(int qlen, int tlen, int w);

// Builds the strip geometry, waves (each wave's boundary columns plus its traceback arena
// under tb_budget bytes) and the processing order of the given pairs.  A pair that cannot
// run within the budget even with its traceback recomputed group by group (Singletrack
// pairs cannot be split) is appended to *refused and left out of the plan; with refused ==
// nullptr the build fails with AW_E_NOMEM_INTERNAL instead.
int band_plan_build(BandPlan &bp, const std::vector<int32_t> &ids, const std::vector<int> &qlen,
                    const std::vector<int> &tlen, const std::vector<int> &w, const std::vector<KswPair> &pairs,
                    int flag, int block, int64_t tb_budget, int nc, std::vector<int32_t> *refused);

// Progress counters sit one 128-byte line apart (one line per strip).
constexpr int PROG_STRIDE = 32;

struct BandDev {
    BandPairDev *pairs;
    BandStripDev *strips;
    int2 *units;
    BandRes *res;
    BandWalkState *walk;  // per pair slot
    int32_t *progress;  // one counter per strip descriptor, PROG_STRIDE ints apart
    int32_t *queue;     // one counter per wave, 64 ints apart
    uint2 *bnd;
    uint8_t *tb;
    int32_t *error;
    const unsigned long long *deadline = nullptr;  // the calling thread's deadline word, or null
    const BandGroupDev *groups = nullptr;          // the group table of the recompute rounds
};

int band_occupancy(int flag);

// Enqueues wave k's counter resets and DP kernel.
cudaError_t band_launch_dp(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                           const uint8_t *tcodes, const KswScore &S, int flag, int ctas, cudaStream_t st);
// Enqueues wave k's result records and tracebacks (one warp per pair).
cudaError_t band_launch_finish(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                               const uint8_t *tcodes, const KswScore &S, int flag, KswOut *out, uint32_t *cig,
                               const int8_t *mat, int m, cudaStream_t st);
// Enqueues the recompute rounds of wave k's recomputed pairs: per round, the strips of one
// group of every such pair again with their traceback stored, then the walks through them.
cudaError_t band_launch_groups(const BandPlan &bp, int k, const BandDev &D, const uint8_t *qcodes,
                               const uint8_t *tcodes, const KswScore &S, int flag, KswOut *out, uint32_t *cig,
                               const int8_t *mat, int m, int ctas, cudaStream_t st);

}  // namespace aw
