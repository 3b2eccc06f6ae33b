// Warp-cooperative traceback reads for the strip layouts.
//
// A traceback walk (ksw_backtrack, the Singletrack reconstruction) is a chain of
// dependent one-byte reads that move up and left through the matrix; read one by
// one from HBM each costs a full memory latency.  Here all 32 lanes of a warp run
// the same walk in lockstep (the walk is uniform), and a miss makes the warp fetch
// a whole tile of lane-words around the missing cell in one parallel round:
// TR rows (or anti-diagonals) x TG column groups of 8 target columns, the rows and
// groups at and before the miss, which is where the walk goes next.  Two tile slots, so the
// vertical and horizontal probes of a Singletrack gap search stay cached together.
#pragma once
#include <stdint.h>
#include <climits>
#include <type_traits>

namespace aw {

// WB: bytes per lane-word, 4 or 8 (state bytes) or 16 (Singletrack v|u tracks); a tile is
// TR_ rows (matrix rows, or anti-diagonals for the anti-diagonal layout) x TG_ groups.
template <int WB, int TR_ = 32, int TG_ = 8>
struct TileCache {
    static constexpr int TR = TR_, TG = TG_, NW = TR * TG;
    using Word = typename std::conditional<WB == 16, uint4,
                                           typename std::conditional<WB == 8, uint2, uint32_t>::type>::type;
    Word *slot[2];  // shared memory, NW words each
    int g0[2], j0[2];
    int next;

    __device__ void init(Word *smem) {
        slot[0] = smem, slot[1] = smem + NW;
        g0[0] = g0[1] = INT_MIN / 2, j0[0] = j0[1] = INT_MIN / 2;
        next = 0;
    }

    // Byte c (0..WB-1) of the lane-word covering column group g = i >> 3 and row j.
    // LOAD(g, j) returns the word (zero when the cell is not stored).
    template <class LOAD>
    __device__ uint32_t byte(int g, int j, int c, LOAD &&load) {
        int k = -1;
#pragma unroll
        for (int t = 0; t < 2; ++t)
            if (g <= g0[t] && g > g0[t] - TG && j <= j0[t] && j > j0[t] - TR) k = t;
        if (k < 0) {  // uniform across the warp: every lane runs the same walk
            k = next;
            next ^= 1;
            g0[k] = g, j0[k] = j;
            const int lane = threadIdx.x & 31;
            Word *dst = slot[k];
            __syncwarp();
#pragma unroll 4
            for (int w = lane; w < NW; w += 32) dst[w] = load(g - (w % TG), j - (w / TG));
            __syncwarp();
        }
        const Word wd = slot[k][(j0[k] - j) * TG + (g0[k] - g)];
        uint32_t x;
        if (WB == 16) {
            const uint4 &q = reinterpret_cast<const uint4 &>(wd);
            x = c < 4 ? q.x : c < 8 ? q.y : c < 12 ? q.z : q.w;
        } else if (WB == 8) {
            const uint2 &q = reinterpret_cast<const uint2 &>(wd);
            x = c < 4 ? q.x : q.y;
        } else {
            x = reinterpret_cast<const uint32_t &>(wd);
        }
        return (x >> (8 * (c & 3))) & 0xffu;
    }
};

}  // namespace aw
