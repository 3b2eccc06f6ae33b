// Gap-affine-2p end-to-end WFA (WFA2-lib as AnchorWave configures it:
// src/myImportandFunction/WfaAlignment.cpp:143-170) on sm_100a.
//
// One warp per pair; the lanes cover the diagonals of a wavefront.  Per score s:
//   * extend M[s] (wavefront/wavefront_extend.c:86-121): each lane advances its
//     diagonal by comparing 32 bases of pattern and text at a time in 2-bit copies of
//     the sequences (one XOR and __ffsll per 32 bases; the run also ends at the end of
//     either sequence); pairs with any byte other than A, C, G, T (the reference compares
//     raw characters) compare 8 bytes at a time instead, where the sentinels after each
//     sequence ('!' pattern, '?' text, wavefront/wavefront_sequences.c:37-39) stop the run;
//   * end-to-end check on diagonal tlen-plen (wavefront/wavefront_termination.c:37-60);
//   * compute s+1 from M[s-x], M[s-o1-e1], I1/D1[s-e1], M[s-o2-e2], I2/D2[s-e2]
//     (wavefront/wavefront_compute_affine2p.c:45-106) over the limits of
//     wavefront/wavefront_compute.c:56-105 (a missing input counts as the null
//     wavefront lo=1, hi=-1), allocating I/D outputs only when one of their
//     inputs exists (:459-572), then trimming out-of-matrix ends (:654-690).
// Values outside a wavefront's trimmed [lo, hi] read as NULL, which is what the
// reference's NULL end padding gives.  Standard mode retains every component of
// every score for the piggyback backtrace (wavefront/wavefront_backtrace.c:321-530);
// Singletrack keeps only M and recycles I/D through a ring of max(e1,e2)+1 slots,
// then reconstructs the path from M (:587-762).
// Medium and low memory (the piggyback modes, wavefront/wavefront_compute_affine2p.c:110-282)
// keep only the scores the compute step still reads (M: the last max_score_scope; I1/D1:
// the last e1+1; I2/D2: the last e2+1) in rings of slots; every cell carries the
// packed CIGAR of its latest operations and a link to the block that holds the earlier
// ones, and a cell whose packed CIGAR reaches 15 operations moves it into a new block
// (wavefront/wavefront_backtrace_offload.c); the traceback follows the links from the end
// cell and unpacks the blocks oldest first, re-extending the matches
// (wavefront/wavefront_backtrace.c:767-799, wavefront/wavefront_pcigar.c:222-278).
//
// Memory: per-score headers and wavefront arrays come from one device pool by a
// bump allocator (atomicAdd, 256 KiB chunks).  A pair that finds the pool empty
// stops with WFA_RETRY and the host re-runs it in a later round with a fresh pool.
#include "aw_internal.h"
#include "wfa_internal.h"

#include <cooperative_groups.h>

namespace aw {
namespace {

constexpr int32_t WF_NULL = INT32_MIN / 2;
constexpr int HDR_CHUNK = 256;               // scores per header chunk
constexpr int64_t DATA_CHUNK = 256 << 10;    // bytes per data chunk

struct CompHdr {
    int32_t lo, hi, base, pad;
    int64_t off;  // byte offset of offsets[base] in the pool
};
struct ScoreHdr {
    CompHdr c[5];  // M, I1, D1, I2, D2
};
enum { CM = 0, CI1 = 1, CD1 = 2, CI2 = 3, CD2 = 4 };

struct Alloc {
    int64_t cur, end;
    bool ok;
    int64_t used;  // bytes taken from the pool (lane 0's copy)
};

// Packed CIGAR of the piggyback modes (wavefront/wavefront_pcigar.h:44-71): 2 bits per
// operation, newest lowest (1 deletion, 2 mismatch or gap close, 3 insertion).
constexpr uint32_t PC_ALMOST_FULL = 0x10000000u;  // 15 operations or more
constexpr uint32_t BT_NULL = 0xFFFFFFFFu;          // no earlier block
constexpr int PIG_U = 2;                           // diagonals per lane in flight
constexpr uint32_t LANE_BLOCKS = 32;               // blocks a lane reserves at a time

__device__ __forceinline__ int64_t pool_grab(const WfaArgs &A, int64_t bytes) {
    const unsigned long long b = atomicAdd(A.pool_head, (unsigned long long)bytes);
    if ((int64_t)(b + bytes) > A.pool_bytes) return -1;
    return (int64_t)b;
}

// Lane-0 bump allocation inside the warp's current chunk; broadcast to the warp.
__device__ int64_t warp_alloc(const WfaArgs &A, Alloc &al, int64_t bytes, int lane) {
    bytes = (bytes + 15) & ~(int64_t)15;
    int64_t r = -1;
    if (lane == 0) {
        if (al.ok) {
            if (al.cur + bytes > al.end) {
                const int64_t sz = bytes > DATA_CHUNK ? bytes : DATA_CHUNK;
                const int64_t b = pool_grab(A, sz);
                if (b < 0) al.ok = false;
                else al.cur = b, al.end = b + sz, al.used += sz;
            }
            if (al.ok) {
                r = al.cur;
                al.cur += bytes;
            }
        }
    }
    r = __shfl_sync(0xffffffffu, r, 0);
    al.ok = __shfl_sync(0xffffffffu, al.ok ? 1 : 0, 0);
    al.cur = __shfl_sync(0xffffffffu, al.cur, 0);
    al.end = __shfl_sync(0xffffffffu, al.end, 0);
    return r;
}

__device__ __forceinline__ ScoreHdr *hdr_ptr(const WfaArgs &A, const int64_t *ctab, int s) {
    return (ScoreHdr *)(A.pool + ctab[s / HDR_CHUNK]) + (s % HDR_CHUNK);
}

// The forward pass reads the headers of the last max_score_scope scores only; each warp
// keeps them in a shared-memory ring of RS (a power of two above the scope) as well as in
// the pool (the backtrace reads all of them from the pool).  RS = 0: pool only.
struct HdrRing {
    ScoreHdr *ring;
    int rs;
    __device__ __forceinline__ const ScoreHdr *get(const WfaArgs &A, const int64_t *ctab, int sc, int s) const {
        if (rs && sc > s - rs) return ring + (sc & (rs - 1));
        return hdr_ptr(A, ctab, sc);
    }
};

__device__ __forceinline__ int32_t getv(const WfaArgs &A, const CompHdr &h, int k) {
    if (k < h.lo || k > h.hi) return WF_NULL;
    return ((const int32_t *)(A.pool + h.off))[k - h.base];
}

// An input wavefront of the compute step: its range and the address of its diagonal 0 (the
// header's base folded in), so that a lane holds four values per input instead of six.
struct InHdr {
    int lo, hi;
    const int32_t *p;
};
__device__ __forceinline__ InHdr in_hdr(const WfaArgs &A, const CompHdr &h) {
    return InHdr{h.lo, h.hi, (const int32_t *)(A.pool + h.off) - h.base};
}
__device__ __forceinline__ int32_t getv(const InHdr &h, int k) {
    return (k < h.lo || k > h.hi) ? WF_NULL : h.p[k];
}
__device__ __forceinline__ int32_t getv_l2(const InHdr &h, int k) {
    return (k < h.lo || k > h.hi) ? WF_NULL : __ldcg(h.p + k);
}

// A piggyback cell: offset, packed CIGAR, link.  In a ring slot the three arrays of a
// component lie h.pad elements apart.
struct Cell {
    int32_t o;
    uint32_t pc, pv;
};
__device__ __forceinline__ Cell getc(const WfaArgs &A, const CompHdr &h, int k) {
    if (k < h.lo || k > h.hi) return Cell{WF_NULL, 0u, BT_NULL};
    const int32_t *d = (const int32_t *)(A.pool + h.off) + (k - h.base);
    return Cell{d[0], (uint32_t)d[h.pad], (uint32_t)d[2 * h.pad]};
}

__device__ __forceinline__ uint64_t load8(const uint8_t *base, int64_t pos) {
    const uintptr_t a = (uintptr_t)(base + pos);
    const uint64_t *p = (const uint64_t *)(a & ~(uintptr_t)7);
    const int sh = (int)(a & 7) * 8;
    const uint64_t lo = p[0];
    if (!sh) return lo;
    return (lo >> sh) | (p[1] << (64 - sh));
}

// 32 bases from base g of a 2-bit arena (base i at bits 2*(i%32) of word i/32); the arena
// ends with a spare word.
__device__ __forceinline__ uint64_t load32b(const uint64_t *p, int64_t g) {
    const int64_t w = g >> 5;
    const int sh = (int)(g & 31) * 2;
    const uint64_t lo = __ldg(p + w);
    if (!sh) return lo;
    return (lo >> sh) | (__ldg(p + w + 1) << (64 - sh));
}

__device__ __forceinline__ bool in_matrix(int32_t o, int k, int plen, int tlen) {
    return (uint32_t)o <= (uint32_t)tlen && (uint32_t)(o - k) <= (uint32_t)plen;
}

// Length of the run of equal bases from pattern[v] / text[h], by the extend step's rules
// (2-bit words for ACGT-only pairs, else 8 bytes at a time up to the sentinels).
__device__ int64_t lcp1(const WfaArgs &A, const WfaPairDev &PR, const uint8_t *pat, const uint8_t *txt, int64_t v,
                        int64_t h) {
    const int64_t rem = min((int64_t)PR.plen - v, (int64_t)PR.tlen - h);
    if (rem <= 0) return 0;
    int64_t n = 0;
    if (PR.packed) {
        for (;;) {
            const uint64_t x = load32b(A.ppat, PR.poff + v + n) ^ load32b(A.ptxt, PR.toff + h + n);
            n += x ? (int64_t)((__ffsll((long long)x) - 1) >> 1) : 32;
            if (x || n >= rem) return min(n, rem);
        }
    }
    for (;;) {
        const uint64_t x = load8(pat, v + n) ^ load8(txt, h + n);
        if (x) return n + ((__ffsll((long long)x) - 1) >> 3);
        n += 8;
    }
}

__device__ __forceinline__ int64_t pb(int32_t o, int t) {
    return (int64_t)((((uint64_t)(int64_t)o) << 4) | (uint64_t)t);
}

struct OpsWriter {
    char *buf;
    int n, cap;
    bool ok;
    __device__ void put(char c, int times) {
        for (int i = 0; i < times; ++i) {
            if (n >= cap) { ok = false; return; }
            buf[n++] = c;
        }
    }
};

// Extends N diagonals of one lane at once (wavefront/wavefront_extend.c:86-121): o[u] is the
// offset on diagonal k0 + stride*u (WF_NULL: nothing to extend) and becomes the offset after the run
// of equal bases.  2-bit words (32 bases per XOR) for ACGT-only pairs; otherwise 8 bytes per
// XOR up to the sentinels after each sequence.  The N loads of a round are in flight together.
template <int N>
__device__ __forceinline__ bool any_of(const bool (&r)[N]) {
    bool a = false;
#pragma unroll
    for (int u = 0; u < N; ++u) a |= r[u];
    return a;
}

template <int N>
__device__ __forceinline__ void extend_n(const WfaArgs &A, const WfaPairDev &PR, const uint8_t *pat,
                                         const uint8_t *txt, int k0, int stride, int32_t (&o)[N]) {
    // o[u] is the text position h; the pattern position is h - k
    const int plen = PR.plen, tlen = PR.tlen;
    bool run[N];
#pragma unroll
    for (int u = 0; u < N; ++u) run[u] = o[u] != WF_NULL;
    bool any = any_of(run);
    if (PR.packed) {
        // 32 bases per XOR; the run ends at the first differing base or at the end of either
        // sequence (the sentinels of the byte path)
#pragma unroll
        for (int u = 0; u < N; ++u)
            if (run[u] && min(plen - (o[u] - (k0 + stride * u)), tlen - o[u]) <= 0) run[u] = false;
        any = any_of(run);
        while (any) {
            uint64_t x[N];
#pragma unroll
            for (int u = 0; u < N; ++u)
                x[u] = run[u] ? (load32b(A.ppat, PR.poff + (o[u] - (k0 + stride * u))) ^ load32b(A.ptxt, PR.toff + o[u]))
                              : 0;
            any = false;
#pragma unroll
            for (int u = 0; u < N; ++u) {
                if (!run[u]) continue;
                const int rem = min(plen - (o[u] - (k0 + stride * u)), tlen - o[u]);
                int nb = x[u] ? (__ffsll((long long)x[u]) - 1) >> 1 : 32;
                const bool stop = x[u] != 0 || nb >= rem;
                if (nb > rem) nb = rem;
                o[u] += nb;
                if (stop || rem == nb) run[u] = false;
                else any = true;
            }
        }
        return;
    }
    while (any) {
        uint64_t x[N];
#pragma unroll
        for (int u = 0; u < N; ++u) x[u] = run[u] ? (load8(pat, o[u] - (k0 + stride * u)) ^ load8(txt, o[u])) : 0;
        any = false;
#pragma unroll
        for (int u = 0; u < N; ++u) {
            if (!run[u]) continue;
            if (x[u]) {
                o[u] += (__ffsll((long long)x[u]) - 1) >> 3;
                run[u] = false;
            } else {
                o[u] += 8;
                any = true;
            }
        }
    }
}

// The result of one pair (one thread): the backtrace of a pair that reached the end
// (status 0), the CIGAR operations reversed into forward order, and the output record.
template <bool PIG>
__device__ void finish_pair(const WfaArgs &A, const WfaPairDev &PR, int idx, const uint8_t *pat, const uint8_t *txt,
                            const int64_t *ctab, const HdrRing &HR, int status, int end_score, int s, int64_t used) {
    const WfaPen P = A.pen;
    const int plen = PR.plen, tlen = PR.tlen;
    const int k_end = tlen - plen;
    WfaOutDev o;
    o.status = status, o.score = 0, o.n_ops = 0, o.final_s = s;
    o.mem_bytes = used;
    if (status == 0) {
        OpsWriter w{A.ops + PR.ops_off, 0, plen + tlen + 8, true};
        if constexpr (PIG) {
            // reverse the links from the end cell in place, then unpack the blocks
            // oldest first: before every operation taken in M the run of matches
            // is re-extended; the mismatch that closes a gap is dropped
            const CompHdr m = HR.get(A, ctab, end_score, end_score)->c[CM];
            const uint32_t *md = (const uint32_t *)(A.pool + m.off) + (k_end - m.base);
            const uint32_t pc_end = md[m.pad];
            uint32_t cur = md[2 * m.pad], prv = BT_NULL;
            uint2 *blk = (uint2 *)A.pool;
            const int64_t lim = 2 * ((int64_t)plen + tlen) + 64;
            int64_t steps = 0;
            bool ok = true;
            while (cur != BT_NULL) {
                if (++steps > lim) { ok = false; break; }
                const uint32_t nxt = blk[cur].y;
                blk[cur].y = prv;
                prv = cur, cur = nxt;
            }
            int64_t v = 0, h = 0;
            bool in_m = true;
            cur = prv;
            for (bool last = false; ok && !last;) {
                uint32_t pc;
                if (cur != BT_NULL) pc = blk[cur].x, cur = blk[cur].y;
                else pc = pc_end, last = true;
                const int len = pc ? 16 - (__clz(pc) >> 1) : 0;
                for (int j = len - 1; j >= 0; --j) {
                    if (in_m) {
                        const int64_t nm = lcp1(A, PR, pat, txt, v, h);
                        w.put('M', (int)nm);
                        v += nm, h += nm;
                    }
                    const uint32_t op = (pc >> (2 * j)) & 3u;
                    if (!in_m && op == 2u) {
                        in_m = true;
                        continue;
                    }
                    w.put(op == 1u ? 'D' : op == 2u ? 'X' : 'I', 1);
                    v += (op == 1u || op == 2u), h += (op == 2u || op == 3u);
                    in_m = op == 2u;
                    if (op == 0u || v > plen || h > tlen) { ok = false; break; }
                }
            }
            if (ok) {
                const int64_t nm = min((int64_t)plen - v, (int64_t)tlen - h);
                w.put('M', (int)nm);
                v += nm, h += nm;
                w.put('I', (int)(tlen - h));
                w.put('D', (int)(plen - v));
            } else {
                o.status = WFA_UNATTAINABLE;
            }
        } else if (!A.singletrack) {
            enum { BM = 9, BD2E = 8, BD2O = 7, BD1E = 6, BD1O = 5, BI2E = 4, BI2O = 3, BI1E = 2, BI1O = 1 };
            int mt = CM, sc = end_score, k = k_end;
            int32_t off = tlen;
            int v = off - k, h = off;
            const int64_t NEG = pb(WF_NULL, 0);
            while (v > 0 && h > 0 && sc > 0) {
                const int smm = sc - P.x, sg1 = sc - P.o1 - P.e1, sg2 = sc - P.o2 - P.e2, sx1 = sc - P.e1,
                          sx2 = sc - P.e2;
                auto G = [&](int scr, int comp, int kk, int add, int t) -> int64_t {
                    if (scr < 0) return NEG;
                    const CompHdr hh = hdr_ptr(A, ctab, scr)->c[comp];
                    return pb(getv(A, hh, kk) + add, t);
                };
                int64_t mall;
                const int64_t i1o = (mt == CM || mt == CI1) ? G(sg1, CM, k - 1, 1, BI1O) : NEG;
                const int64_t i1e = (mt == CM || mt == CI1) ? G(sx1, CI1, k - 1, 1, BI1E) : NEG;
                const int64_t d1o = (mt == CM || mt == CD1) ? G(sg1, CM, k + 1, 0, BD1O) : NEG;
                const int64_t d1e = (mt == CM || mt == CD1) ? G(sx1, CD1, k + 1, 0, BD1E) : NEG;
                const int64_t i2o = (mt == CM || mt == CI2) ? G(sg2, CM, k - 1, 1, BI2O) : NEG;
                const int64_t i2e = (mt == CM || mt == CI2) ? G(sx2, CI2, k - 1, 1, BI2E) : NEG;
                const int64_t d2o = (mt == CM || mt == CD2) ? G(sg2, CM, k + 1, 0, BD2O) : NEG;
                const int64_t d2e = (mt == CM || mt == CD2) ? G(sx2, CD2, k + 1, 0, BD2E) : NEG;
                if (mt == CM) {
                    const int64_t misms = G(smm, CM, k, 1, BM);
                    mall = max(misms, max(max(max(i1o, i1e), max(i2o, i2e)), max(max(d1o, d1e), max(d2o, d2e))));
                } else if (mt == CI1) mall = max(i1o, i1e);
                else if (mt == CI2) mall = max(i2o, i2e);
                else if (mt == CD1) mall = max(d1o, d1e);
                else mall = max(d2o, d2e);
                if (mall < 0) break;
                if (mt == CM) {
                    const int mo = (int)(mall >> 4);
                    w.put('M', off - mo);
                    off = mo;
                    v = off - k, h = off;
                    if (v <= 0 || h <= 0) break;
                }
                const int bt = (int)(mall & 0xf);
                switch (bt) {
                case BM: sc = smm; mt = CM; break;
                case BI1O: sc = sg1; mt = CM; break;
                case BI1E: sc = sx1; mt = CI1; break;
                case BI2O: sc = sg2; mt = CM; break;
                case BI2E: sc = sx2; mt = CI2; break;
                case BD1O: sc = sg1; mt = CM; break;
                case BD1E: sc = sx1; mt = CD1; break;
                case BD2O: sc = sg2; mt = CM; break;
                default: sc = sx2; mt = CD2; break;
                }
                if (bt == BM) w.put('X', 1), --off;
                else if (bt <= BI2E) w.put('I', 1), --k, --off;
                else w.put('D', 1), ++k;
                v = off - k, h = off;
            }
            if (mt == CM) {
                if (v > 0 && h > 0) {
                    const int nm = v < h ? v : h;
                    w.put('M', nm);
                    v -= nm, h -= nm;
                }
                w.put('D', v > 0 ? v : 0);
                w.put('I', h > 0 ? h : 0);
            }
        } else {
            int sc = end_score, k = k_end, gl = 0;
            bool in_m = true, ok = true;
            int32_t off = tlen, off_be = off;
            const int64_t maxgap = (int64_t)plen + tlen;
            while (sc != 0) {
                if (sc < 0 || off < 0) { ok = false; break; }
                if (in_m) {
                    const int v = off - k, h = off;
                    if (v < 0 || h < 0 || v > plen || h > tlen) { ok = false; break; }
                    int nm = 0;
                    while (nm < v && nm < h && pat[v - nm - 1] == txt[h - nm - 1]) ++nm;
                    off_be = off - nm;
                    const int ms = sc - P.x;
                    bool took = false;
                    if (ms >= 0) {
                        const CompHdr mh = hdr_ptr(A, ctab, ms)->c[CM];
                        if (mh.lo <= k && k <= mh.hi &&
                            ((const int32_t *)(A.pool + mh.off))[k - mh.base] + 1 == off_be) {
                            w.put('M', nm);
                            w.put('X', 1);
                            off = off_be - 1;
                            sc = ms;
                            took = true;
                        }
                    }
                    if (!took) in_m = false, gl = 0;
                    continue;
                }
                ++gl;
                if ((int64_t)gl > maxgap) { ok = false; break; }
                const int ki = k - gl, kd = k + gl;
                for (int piece = 0; piece < 2; ++piece) {
                    const int64_t isc = piece == 0 ? (int64_t)sc - P.o1 - (int64_t)gl * P.e1
                                                   : (int64_t)sc - P.o2 - (int64_t)gl * P.e2;
                    if (isc < 0 || isc > s) continue;
                    const CompHdr ih = hdr_ptr(A, ctab, (int)isc)->c[CM];
                    const int32_t *id = (const int32_t *)(A.pool + ih.off);
                    if (ih.lo <= ki && ki <= ih.hi && id[ki - ih.base] + gl >= off_be &&
                        id[ki - ih.base] + gl <= off) {
                        w.put('M', off - (id[ki - ih.base] + gl));
                        w.put('I', gl);
                        k = ki, off = id[ki - ih.base], sc = (int)isc, in_m = true;
                        break;
                    }
                    if (ih.lo <= kd && kd <= ih.hi && id[kd - ih.base] >= off_be && id[kd - ih.base] <= off) {
                        w.put('M', off - id[kd - ih.base]);
                        w.put('D', gl);
                        k = kd, off = id[kd - ih.base], sc = (int)isc, in_m = true;
                        break;
                    }
                }
            }
            if (ok && (!in_m || k != 0 || off < 0 || off > plen || off > tlen)) ok = false;
            if (ok)
                for (int i = 0; i < off; ++i)
                    if (pat[i] != txt[i]) { ok = false; break; }
            if (ok) w.put('M', off);
            if (!ok) o.status = WFA_UNATTAINABLE;
        }
        if (!w.ok) o.status = WFA_OVERFLOW;
        if (o.status == 0) {
            for (int a = 0, b = PIG ? 0 : w.n - 1; a < b; ++a, --b) {
                const char t = w.buf[a];
                w.buf[a] = w.buf[b], w.buf[b] = t;
            }
            o.score = -end_score;
            o.n_ops = w.n;
        }
    }
    A.out[idx] = o;
}

// One trip of the piggyback compute step over the diagonals kb + g0 + G*u (u < PIG_U) of a
// score with range [lo, hi], inputs in[] (M[s-x], M[s-o1-e1], I1[s-e1], D1[s-e1], M[s-o2-e2],
// I2[s-e2], D2[s-e2]) and outputs out[] (ring slots of rcap elements per array).  Each gap cell
// takes the extension on a tie, M the mismatch, then D2, D1, I2, I1 (the kernel's assignment
// order); M is extended as it is computed (matches are not recorded in the packed CIGAR; the
// traceback re-extends them).  Cells whose packed CIGAR holds 15 operations move it into a
// block from the lane's reserved run; lanes whose run is short reserve LANE_BLOCKS more in one
// allocation of the warp (`wal`).  Every lane of the warp must call it.  Returns false when
// the pool is exhausted.
__device__ __forceinline__ bool pig_trip(const WfaArgs &A, const WfaPairDev &PR, const uint8_t *pat,
                                         const uint8_t *txt, int kb, int g0, int G, int lo, int hi,
                                         const CompHdr (&in)[7], const CompHdr (&out)[5], int mask, int rcap,
                                         Alloc &wal, uint32_t &bnext, uint32_t &bend, int (&kmin)[5], int (&kmax)[5],
                                         bool &reached) {
    const int plen = PR.plen, tlen = PR.tlen, k_end = tlen - plen, lane = threadIdx.x & 31;
    const CompHdr &m_misms = in[0], &m_open1 = in[1], &i1 = in[2], &d1 = in[3], &m_open2 = in[4], &i2 = in[5],
                  &d2 = in[6];
    const int k0 = kb + g0;
    Cell C[PIG_U][5];
#pragma unroll
    for (int u = 0; u < PIG_U; ++u) {
        const int k = k0 + G * u;
        Cell a = getc(A, m_open1, k - 1), b = getc(A, i1, k - 1);
        Cell g = b.o >= a.o ? b : a;
        C[u][CI1] = Cell{g.o + 1, (g.pc << 2) | 3u, g.pv};
        a = getc(A, m_open2, k - 1), b = getc(A, i2, k - 1);
        g = b.o >= a.o ? b : a;
        C[u][CI2] = Cell{g.o + 1, (g.pc << 2) | 3u, g.pv};
        a = getc(A, m_open1, k + 1), b = getc(A, d1, k + 1);
        g = b.o >= a.o ? b : a;
        C[u][CD1] = Cell{g.o, (g.pc << 2) | 1u, g.pv};
        a = getc(A, m_open2, k + 1), b = getc(A, d2, k + 1);
        g = b.o >= a.o ? b : a;
        C[u][CD2] = Cell{g.o, (g.pc << 2) | 1u, g.pv};
        Cell x = getc(A, m_misms, k);
        x.o += 1;
        const int32_t best = max(max(C[u][CD1].o, C[u][CD2].o), max(x.o, max(C[u][CI1].o, C[u][CI2].o)));
        const Cell &src = best == x.o ? x
                          : best == C[u][CD2].o ? C[u][CD2]
                          : best == C[u][CD1].o ? C[u][CD1]
                          : best == C[u][CI2].o ? C[u][CI2]
                                                : C[u][CI1];
        C[u][CM] = Cell{in_matrix(best, k, plen, tlen) ? best : WF_NULL, (src.pc << 2) | 2u, src.pv};
    }
    {
        int32_t mo[PIG_U];
#pragma unroll
        for (int u = 0; u < PIG_U; ++u) mo[u] = k0 + G * u <= hi ? C[u][CM].o : WF_NULL;
        extend_n<PIG_U>(A, PR, pat, txt, k0, G, mo);
#pragma unroll
        for (int u = 0; u < PIG_U; ++u) {
            const int k = k0 + G * u;
            if (k > hi) continue;
            C[u][CM].o = mo[u];
            if (k == k_end && mo[u] != WF_NULL && mo[u] >= tlen) reached = true;
        }
    }
    uint32_t fl = 0;
#pragma unroll
    for (int u = 0; u < PIG_U; ++u) {
        const int k = k0 + G * u;
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (k <= hi && (mask & (1 << c)) && C[u][c].pc >= PC_ALMOST_FULL && in_matrix(C[u][c].o, k, plen, tlen))
                fl |= 1u << (u * 5 + c);
    }
    const bool refill = bend - bnext < (uint32_t)__popc(fl);
    const unsigned rb = __ballot_sync(0xffffffffu, refill);
    if (rb) {
        const int64_t bb = warp_alloc(A, wal, (int64_t)__popc(rb) * LANE_BLOCKS * 8, lane);
        if (bb < 0) return false;
        if (refill) {
            bnext = (uint32_t)(bb >> 3) + (uint32_t)__popc(rb & ((1u << lane) - 1u)) * LANE_BLOCKS;
            bend = bnext + LANE_BLOCKS;
        }
    }
    if (fl) {
        uint2 *blk = (uint2 *)A.pool;
#pragma unroll
        for (int u = 0; u < PIG_U; ++u)
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (fl & (1u << (u * 5 + c))) {
                    blk[bnext] = make_uint2(C[u][c].pc, C[u][c].pv);
                    C[u][c].pc = 0u, C[u][c].pv = bnext++;
                }
    }
#pragma unroll
    for (int u = 0; u < PIG_U; ++u) {
        const int k = k0 + G * u;
        if (k > hi) break;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            if (!(mask & (1 << c))) continue;
            int32_t *d = (int32_t *)(A.pool + out[c].off) + (k - lo);
            d[0] = C[u][c].o, d[rcap] = (int32_t)C[u][c].pc, d[2 * rcap] = (int32_t)C[u][c].pv;
            if (in_matrix(C[u][c].o, k, plen, tlen)) kmin[c] = min(kmin[c], k), kmax[c] = max(kmax[c], k);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// Plans and partials shared by the CTA-cooperative mode below and the cluster kernel: the
// plan of one score (its range, inputs and outputs) and, per CTA, the trimmed ends of each
// component and whether the end cell was reached.
enum { WOP_COMPUTE = 0, WOP_DONE = 1, WOP_EXIT = 2 };

struct WidePlan {
    int op, lo, hi, mask;  // mask: components allocated at the planned score (bit c)
    CompHdr in[7];         // M[s-x], M[s-o1-e1], I1[s-e1], D1[s-e1], M[s-o2-e2], I2[s-e2], D2[s-e2]
    CompHdr out[5];
};
struct WidePart {
    int kmin[5], kmax[5], reached, pad;
    int retry, pad2;          // a warp found the pool exhausted (CTA-cooperative piggyback mode)
    unsigned long long used;  // pool bytes of the warps' block reservations (the same)
};

__device__ __forceinline__ void part_reset(WidePart &p) {
    for (int c = 0; c < 5; ++c) p.kmin[c] = INT_MAX, p.kmax[c] = INT_MIN;
    p.reached = 0;
}

// The input headers of score s from the header ring (null below score 0).
__device__ __forceinline__ void plan_inputs(const WfaArgs &A, const int64_t *ctab, const HdrRing &HR, int s,
                                            CompHdr (&in)[7]) {
    const WfaPen P = A.pen;
    const CompHdr NUL{1, -1, 0, 0, 0};
    const int sm = s - P.x, so1 = s - P.o1 - P.e1, se1 = s - P.e1, so2 = s - P.o2 - P.e2, se2 = s - P.e2;
    in[0] = sm >= 0 ? HR.get(A, ctab, sm, s)->c[CM] : NUL;
    in[1] = so1 >= 0 ? HR.get(A, ctab, so1, s)->c[CM] : NUL;
    in[2] = se1 >= 0 ? HR.get(A, ctab, se1, s)->c[CI1] : NUL;
    in[3] = se1 >= 0 ? HR.get(A, ctab, se1, s)->c[CD1] : NUL;
    in[4] = so2 >= 0 ? HR.get(A, ctab, so2, s)->c[CM] : NUL;
    in[5] = se2 >= 0 ? HR.get(A, ctab, se2, s)->c[CI2] : NUL;
    in[6] = se2 >= 0 ? HR.get(A, ctab, se2, s)->c[CD2] : NUL;
}

// The limits of the compute step over its inputs (null inputs contribute lo=1, hi=-1) and
// which I/D outputs exist (one of their inputs exists).
__device__ __forceinline__ void plan_limits(const CompHdr (&in)[7], int &lo, int &hi, int &mask) {
    bool isnull[7];
    for (int j = 0; j < 7; ++j) isnull[j] = in[j].lo > in[j].hi;
    lo = in[0].lo, hi = in[0].hi;
    lo = min(lo, in[1].lo - 1), hi = max(hi, in[1].hi + 1);
    lo = min(lo, in[2].lo + 1), hi = max(hi, in[2].hi + 1);
    lo = min(lo, in[3].lo - 1), hi = max(hi, in[3].hi - 1);
    lo = min(lo, in[4].lo - 1), hi = max(hi, in[4].hi + 1);
    lo = min(lo, in[5].lo + 1), hi = max(hi, in[5].hi + 1);
    lo = min(lo, in[6].lo - 1), hi = max(hi, in[6].hi - 1);
    mask = 1;
    if (!isnull[1] || !isnull[2]) mask |= 1 << CI1;
    if (!isnull[1] || !isnull[3]) mask |= 1 << CD1;
    if (!isnull[4] || !isnull[5]) mask |= 1 << CI2;
    if (!isnull[4] || !isnull[6]) mask |= 1 << CD2;
}

// A warp's trimmed ends and end check, folded into its CTA's partials.
__device__ __forceinline__ void fold_partials(const int (&kmin)[5], const int (&kmax)[5], bool reached, WidePart &pp) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const int th = __reduce_max_sync(0xffffffffu, kmax[c]);
        const int tl = __reduce_min_sync(0xffffffffu, kmin[c]);
        if (lane == 0 && th != INT_MIN) atomicMax(&pp.kmax[c], th), atomicMin(&pp.kmin[c], tl);
    }
    if (__any_sync(0xffffffffu, reached) && lane == 0) pp.reached = 1;
}

// First array of component c at score sc in the piggyback rings: M's last SR scores, then
// I1/D1's last R1, then I2/D2's last R2, three arrays (offsets, packed CIGARs, links) each.
__device__ __forceinline__ int64_t pig_slot(int c, int sc, int SR, int R1, int R2) {
    if (c == CM) return (int64_t)(sc % SR) * 3;
    if (c <= CD1) return 3 * (int64_t)(SR + (sc % R1) * 2 + (c - CI1));
    return 3 * (int64_t)(SR + 2 * R1 + (sc % R2) * 2 + (c - CI2));
}

// Diagonals per thread in flight in the CTA-cooperative compute step (build-time tuning).
#ifndef AW_WFA_CTA_U
#define AW_WFA_CTA_U 2
#endif

// One thread's diagonals lo + g0 + G*u of a planned score (high memory): the compute step,
// the fused extension of M, the stores, and this thread's trimmed ends and end check, folded
// per warp into the CTA's partials.  `ld_l2` reads the inputs through L2 (other CTAs wrote them).
template <bool L2>
__device__ __forceinline__ void plan_compute(const WfaArgs &A, const WfaPairDev &PR, const uint8_t *pat,
                                             const uint8_t *txt, const WidePlan &Q, int g0, int G, WidePart &pp) {
    const int plen = PR.plen, tlen = PR.tlen, k_end = tlen - plen;
    const int lo = Q.lo, hi = Q.hi, mask = Q.mask;
    const InHdr m_misms = in_hdr(A, Q.in[0]), m_open1 = in_hdr(A, Q.in[1]), i1 = in_hdr(A, Q.in[2]),
                d1 = in_hdr(A, Q.in[3]), m_open2 = in_hdr(A, Q.in[4]), i2 = in_hdr(A, Q.in[5]),
                d2 = in_hdr(A, Q.in[6]);
    int32_t *oM = (int32_t *)(A.pool + Q.out[CM].off);
    int32_t *oI1 = (mask & 2) ? (int32_t *)(A.pool + Q.out[CI1].off) : nullptr;
    int32_t *oD1 = (mask & 4) ? (int32_t *)(A.pool + Q.out[CD1].off) : nullptr;
    int32_t *oI2 = (mask & 8) ? (int32_t *)(A.pool + Q.out[CI2].off) : nullptr;
    int32_t *oD2 = (mask & 16) ? (int32_t *)(A.pool + Q.out[CD2].off) : nullptr;
    int kmin[5], kmax[5];
    bool reached = false;
#pragma unroll
    for (int c = 0; c < 5; ++c) kmin[c] = INT_MAX, kmax[c] = INT_MIN;
    constexpr int U = L2 ? 4 : AW_WFA_CTA_U;
    for (int k0 = lo + g0; k0 <= hi; k0 += G * U) {
        int32_t ins1[U], ins2[U], del1[U], del2[U], misms[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + G * u;
            if constexpr (L2) {
                ins1[u] = max(getv_l2(m_open1, k - 1), getv_l2(i1, k - 1)) + 1;
                ins2[u] = max(getv_l2(m_open2, k - 1), getv_l2(i2, k - 1)) + 1;
                del1[u] = max(getv_l2(m_open1, k + 1), getv_l2(d1, k + 1));
                del2[u] = max(getv_l2(m_open2, k + 1), getv_l2(d2, k + 1));
                misms[u] = getv_l2(m_misms, k) + 1;
            } else {
                ins1[u] = max(getv(m_open1, k - 1), getv(i1, k - 1)) + 1;
                ins2[u] = max(getv(m_open2, k - 1), getv(i2, k - 1)) + 1;
                del1[u] = max(getv(m_open1, k + 1), getv(d1, k + 1));
                del2[u] = max(getv(m_open2, k + 1), getv(d2, k + 1));
                misms[u] = getv(m_misms, k) + 1;
            }
        }
        int32_t mo[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + G * u;
            const int32_t best = max(max(del1[u], del2[u]), max(misms[u], max(ins1[u], ins2[u])));
            mo[u] = (k <= hi && in_matrix(best, k, plen, tlen)) ? best : WF_NULL;
            if (k > hi) continue;
            if (oI1) oI1[k - lo] = ins1[u];
            if (oD1) oD1[k - lo] = del1[u];
            if (oI2) oI2[k - lo] = ins2[u];
            if (oD2) oD2[k - lo] = del2[u];
            const int32_t vals[4] = {ins1[u], del1[u], ins2[u], del2[u]};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (in_matrix(vals[c], k, plen, tlen)) kmin[c + 1] = min(kmin[c + 1], k), kmax[c + 1] = max(kmax[c + 1], k);
            if (mo[u] != WF_NULL) kmin[CM] = min(kmin[CM], k), kmax[CM] = max(kmax[CM], k);
        }
        extend_n<U>(A, PR, pat, txt, k0, G, mo);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + G * u;
            if (k > hi) break;
            if (k == k_end && mo[u] != WF_NULL && mo[u] >= tlen) reached = true;
            oM[k - lo] = mo[u];
        }
    }
    fold_partials(kmin, kmax, reached, pp);
}

// Thread-0 bump allocation for the CTA-cooperative mode.
__device__ int64_t cta_alloc(const WfaArgs &A, Alloc &al, int64_t bytes) {
    bytes = (bytes + 15) & ~(int64_t)15;
    if (!al.ok) return -1;
    if (al.cur + bytes > al.end) {
        const int64_t sz = bytes > DATA_CHUNK ? bytes : DATA_CHUNK;
        const int64_t b = pool_grab(A, sz);
        if (b < 0) {
            al.ok = false;
            return -1;
        }
        al.cur = b, al.end = b + sz, al.used += sz;
    }
    const int64_t r = al.cur;
    al.cur += bytes;
    return r;
}

// CTA-cooperative mode: one long pair on all threads of a CTA.  Thread 0 plans
// every score (the headers in the CTA's header ring and the pool, the allocations) and all
// threads compute and extend the diagonals lo + tid + NT*u; two CTA barriers per score.  A
// pair whose wavefront grows too wide stops with WFA_WIDE for the cluster kernel.  The cell arithmetic, the limits, the trimming and the backtrace are the warp's.
// In the piggyback modes every warp reserves its own block runs; no pair moves to the
// cluster kernel.
template <bool PIG>
__device__ void cta_pair(const WfaArgs &A, int idx, const HdrRing &HR, WidePlan &plan, WidePart &part) {
    const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31;
    const WfaPen P = A.pen;
    const WfaPairDev PR = A.pairs[idx];
    const int plen = PR.plen, tlen = PR.tlen;
    const uint8_t *pat = A.pat + PR.poff, *txt = A.txt + PR.toff;
    int64_t *ctab = A.ctab + PR.ctab_off;
    const CompHdr NUL{1, -1, 0, 0, 0};
    // thread 0's state
    int s = 0, num_null = 0, status = 0, end_score = -1;
    const int smax = PR.ctab_cap * HDR_CHUNK - 1;
    const int R = (P.e1 > P.e2 ? P.e1 : P.e2) + 1, ring_cap = plen + tlen + 8;
    int64_t ring = -1;
    Alloc al{0, 0, true, 0};
    // piggyback rings (thread 0) and every warp's block reservations
    const int SR = A.max_score_scope, R1 = P.e1 + 1, R2 = P.e2 + 1;
    const int64_t ring_arrays = 3 * (int64_t)(SR + 2 * R1 + 2 * R2);
    int rcap = 32;
    int64_t rbase = -1;
    Alloc wal{0, 0, true, 0};
    uint32_t bnext = 0, bend = 0;
    auto set_hdr = [&](int sc, const CompHdr (&o)[5]) {
        ScoreHdr *OH = hdr_ptr(A, ctab, sc);
        for (int c = 0; c < 5; ++c) OH->c[c] = o[c];
        if (HR.rs)
            for (int c = 0; c < 5; ++c) HR.ring[sc & (HR.rs - 1)].c[c] = o[c];
    };
    auto plan_next = [&]() {
        for (;;) {
            ++s;
            if (s > smax) {
                status = WFA_OVERFLOW;
                break;
            }
            if (s % HDR_CHUNK == 0) {
                const int64_t hb = cta_alloc(A, al, (int64_t)sizeof(ScoreHdr) * HDR_CHUNK);
                if (hb < 0) {
                    status = WFA_RETRY;
                    break;
                }
                ctab[s / HDR_CHUNK] = hb;
            }
            CompHdr in[7];
            plan_inputs(A, ctab, HR, s, in);
            bool all_null = true;
            for (int j = 0; j < 7; ++j) all_null &= in[j].lo > in[j].hi;
            if (all_null) {
                const CompHdr o[5] = {NUL, NUL, NUL, NUL, NUL};
                set_hdr(s, o);
                if (++num_null > A.max_score_scope) {  // the top of the next step: M[s] is empty
                    status = -3;
                    break;
                }
                continue;
            }
            num_null = 0;
            int lo, hi, mask;
            plan_limits(in, lo, hi, mask);
            const int width = hi - lo + 1;
            if constexpr (PIG) {
                if (width > rcap) {
                    const int nc = max(2 * rcap, (width + 3) & ~3);
                    const int64_t nb = cta_alloc(A, al, ring_arrays * nc * 4);
                    if (nb < 0) {
                        status = WFA_RETRY;
                        break;
                    }
                    rcap = nc, rbase = nb;
                }
                for (int c = 0; c < 5; ++c)
                    plan.out[c] = (mask & (1 << c)) ? CompHdr{lo, hi, lo, rcap, rbase + pig_slot(c, s, SR, R1, R2) * rcap * 4}
                                                     : NUL;
                for (int j = 0; j < 7; ++j) plan.in[j] = in[j];
                plan.op = WOP_COMPUTE, plan.lo = lo, plan.hi = hi, plan.mask = mask;
                return;
            }
            // a wavefront too wide for the CTA: the cluster kernel re-runs the pair (past
            // wide_width_cta always; past wide_width_tail in the call's tail, checked every 32
            // scores: every pair started and few still running)
            if (A.wide_width_cta > 0 && width > A.wide_width_tail) {
                bool wide = width > A.wide_width_cta;
                if (!wide && (s & 31) == 0)
                    wide = *(volatile int32_t *)(A.queue + 2) >= A.n_long && *(volatile int32_t *)A.queue >= A.n &&
                           *(volatile int32_t *)(A.queue + 1) <= A.wide_tail_pairs;
                if (wide) {
                    status = WFA_WIDE;
                    break;
                }
            }
            if (A.singletrack && width > ring_cap) {
                status = WFA_OVERFLOW;
                break;
            }
            const int64_t wb = (((int64_t)width * 4) + 15) & ~(int64_t)15;
            const int64_t blk = cta_alloc(A, al, wb * (A.singletrack ? 1 : __popc(mask)));
            if (blk < 0) {
                status = WFA_RETRY;
                break;
            }
            int64_t o = blk;
            for (int c = 0; c < 5; ++c) {
                plan.out[c] = NUL;
                if (!(mask & (1 << c))) continue;
                int64_t place;
                if (c == CM || !A.singletrack) place = o, o += wb;
                else place = ring + ((int64_t)((s % R) * 4 + (c - 1)) * ring_cap) * 4;
                plan.out[c] = CompHdr{lo, hi, lo, 0, place};
            }
            for (int j = 0; j < 7; ++j) plan.in[j] = in[j];
            plan.op = WOP_COMPUTE, plan.lo = lo, plan.hi = hi, plan.mask = mask;
            return;
        }
        plan.op = WOP_DONE;
    };
    if (tid == 0) {
        atomicAdd(A.queue + 1, 1);  // pairs running
        part_reset(part);
        part.retry = 0, part.used = 0;
        if (!PIG && A.singletrack) {
            ring = cta_alloc(A, al, (int64_t)R * 4 * ring_cap * 4);
            if (ring < 0) status = WFA_RETRY;
        }
        if (PIG) {
            rbase = cta_alloc(A, al, ring_arrays * rcap * 4);
            if (rbase < 0) status = WFA_RETRY;
        }
        const int64_t h0 = status == 0 ? cta_alloc(A, al, (int64_t)sizeof(ScoreHdr) * HDR_CHUNK) : -1;
        const int64_t d0 = h0 < 0 ? -1 : PIG ? rbase : cta_alloc(A, al, 16);  // piggyback: slot 0 of M
        if (status == 0 && d0 < 0) status = WFA_RETRY;
        if (status == 0) {
            // M[0] = {0} on diagonal 0, extended
            const int32_t o0 = (int32_t)lcp1(A, PR, pat, txt, 0, 0);
            ctab[0] = h0;
            *(int32_t *)(A.pool + d0) = o0;
            if (PIG) {
                ((uint32_t *)(A.pool + d0))[rcap] = 0u;
                ((uint32_t *)(A.pool + d0))[2 * rcap] = BT_NULL;  // the start (0, 0)
            }
            const CompHdr o[5] = {CompHdr{0, 0, 0, PIG ? rcap : 0, d0}, NUL, NUL, NUL, NUL};
            set_hdr(0, o);
            if (tlen - plen == 0 && o0 >= tlen) end_score = 0;
        }
        if (status != 0 || end_score == 0) plan.op = WOP_DONE;
        else plan_next();
    }
    __syncthreads();
    while (plan.op == WOP_COMPUTE) {
        if constexpr (PIG) {
            int kmin[5], kmax[5];
            bool reached = false, ok = true;
#pragma unroll
            for (int c = 0; c < 5; ++c) kmin[c] = INT_MAX, kmax[c] = INT_MIN;
            for (int kb = plan.lo; kb <= plan.hi && ok; kb += NT * PIG_U)
                ok = pig_trip(A, PR, pat, txt, kb, tid, NT, plan.lo, plan.hi, plan.in, plan.out, plan.mask,
                              plan.out[CM].pad, wal, bnext, bend, kmin, kmax, reached);
            fold_partials(kmin, kmax, reached, part);
            if (!ok && lane == 0) part.retry = 1;
        } else {
            plan_compute<false>(A, PR, pat, txt, plan, tid, NT, part);
        }
        __syncthreads();
        if (tid == 0 && part.retry) {
            status = WFA_RETRY;
            plan.op = WOP_DONE;
        } else if (tid == 0) {
            CompHdr out[5];
            for (int c = 0; c < 5; ++c) {
                out[c] = plan.out[c];
                if (!(plan.mask & (1 << c))) continue;
                // no diagonal in the matrix: the empty range [lo, lo-1] of the scan
                if (part.kmax[c] == INT_MIN) out[c].hi = out[c].lo - 1;
                else out[c].lo = part.kmin[c], out[c].hi = part.kmax[c];
            }
            const bool reached = part.reached != 0;
            part_reset(part);
            set_hdr(s, out);
            if (reached) {
                end_score = s;
                plan.op = WOP_DONE;
            } else {
                plan_next();
            }
        }
        __syncthreads();
    }
    if (PIG && lane == 0) atomicAdd(&part.used, (unsigned long long)wal.used);
    __syncthreads();
    if (tid == 0) {
        finish_pair<PIG>(A, PR, idx, pat, txt, ctab, HR, status, end_score, s, al.used + (int64_t)part.used);
        atomicSub(A.queue + 1, 1);
    }
    __syncthreads();
}

// Build-time tuning of the warp kernel: CTAs per SM the registers are sized for (4 warps
// each), and diagonals per lane in flight in the high-memory compute step.
#ifndef AW_WFA_MINB
#define AW_WFA_MINB 4
#endif
#ifndef AW_WFA_WARP_U
#define AW_WFA_WARP_U 4
#endif
constexpr int WU = AW_WFA_WARP_U;

template <bool PIG>
__global__ void __launch_bounds__(128, AW_WFA_MINB) wfa_kernel(WfaArgs A, int rs) {
    const int lane = threadIdx.x & 31;
    const WfaPen P = A.pen;
    extern __shared__ ScoreHdr hring_all[];
    {
        // the long pairs first, each on the whole CTA (warp 0's header ring serves the
        // planner; the warps take their own rings afterwards)
        __shared__ WidePlan cplan;
        __shared__ WidePart cpart;
        __shared__ int cpi;
        for (;;) {
            if (threadIdx.x == 0) cpi = A.n_long > 0 ? atomicAdd(A.queue + 2, 1) : A.n_long;
            __syncthreads();
            const int pi = cpi;
            __syncthreads();
            if (pi >= A.n_long) break;
            cta_pair<PIG>(A, A.order_long[pi], HdrRing{hring_all, rs}, cplan, cpart);
        }
    }
    const HdrRing HR{hring_all + (threadIdx.x >> 5) * rs, rs};
    for (;;) {
        int pi = 0;
        if (lane == 0) pi = atomicAdd(A.queue, 1);
        pi = __shfl_sync(0xffffffffu, pi, 0);
        if (pi >= A.n) break;
        if (lane == 0) atomicAdd(A.queue + 1, 1);  // pairs running on warps
        const int idx = A.order[pi];
        const WfaPairDev PR = A.pairs[idx];
        const int plen = PR.plen, tlen = PR.tlen;
        const uint8_t *pat = A.pat + PR.poff, *txt = A.txt + PR.toff;
        int64_t *ctab = A.ctab + PR.ctab_off;
        Alloc al{0, 0, true, 0};
        uint32_t bnext = 0, bend = 0;  // this lane's reserved piggyback blocks
        int status = 0, end_score = -1;
        // piggyback rings, each slot three arrays (offsets, packed CIGARs, links) of rcap
        // elements: M keeps its last SR scores, I1/D1 their last e1+1 and I2/D2 their last
        // e2+1 (the only scores the compute step reads them from); grown by reallocation
        const int SR = A.max_score_scope, R1 = P.e1 + 1, R2 = P.e2 + 1;
        const int64_t ring_arrays = 3 * (int64_t)(SR + 2 * R1 + 2 * R2);
        int rcap = 0;
        int64_t rbase = -1;
        if constexpr (PIG) {
            rcap = 32;
            rbase = warp_alloc(A, al, ring_arrays * rcap * 4, lane);
            if (rbase < 0) status = WFA_RETRY;
        }
        // Singletrack ring for I/D: R slots x 4 components x cap offsets
        const int R = (P.e1 > P.e2 ? P.e1 : P.e2) + 1;
        const int ring_cap = plen + tlen + 8;
        int64_t ring = -1;
        if (A.singletrack) {
            ring = warp_alloc(A, al, (int64_t)R * 4 * ring_cap * 4, lane);
            if (ring < 0) status = WFA_RETRY;
        }
        // score 0
        int64_t h0 = -1;
        if (status == 0) {
            h0 = warp_alloc(A, al, (int64_t)sizeof(ScoreHdr) * HDR_CHUNK, lane);
            if (h0 < 0) status = WFA_RETRY;
        }
        int64_t d0 = -1;
        if (status == 0) {
            if constexpr (PIG) d0 = rbase;  // slot 0, component M
            else d0 = warp_alloc(A, al, 16, lane);
            if (d0 < 0) status = WFA_RETRY;
        }
        if (status == 0 && lane == 0) {
            ctab[0] = h0;
            ScoreHdr *H = (ScoreHdr *)(A.pool + h0);
            for (int c = 0; c < 5; ++c) H->c[c] = CompHdr{1, -1, 0, 0, 0};
            H->c[CM] = CompHdr{0, 0, 0, PIG ? rcap : 0, d0};
            *(int32_t *)(A.pool + d0) = 0;
            if constexpr (PIG) {
                ((uint32_t *)(A.pool + d0))[rcap] = 0u;
                ((uint32_t *)(A.pool + d0))[2 * rcap] = BT_NULL;  // the start (0, 0)
            }
            if (HR.rs) HR.ring[0] = *H;
        }
        __syncwarp();
        const int k_end = tlen - plen;
        int s = 0, num_null = 0;
        bool fused_reached = false;  // the compute step's extension reached the end (this lane)
        const int smax = PR.ctab_cap * HDR_CHUNK - 1;
        while (status == 0) {
            // ---- extend M[s] and check the end.  The compute step below extends M[s] as it
            // computes it (fused), so here only M[0] is extended.
            {
                const CompHdr m = HR.get(A, ctab, s, s)->c[CM];
                bool reached = false;
                if (m.lo <= m.hi) {
                    if (s == 0) {
                        int32_t *d = (int32_t *)(A.pool + m.off);
                        for (int k0 = m.lo + lane; k0 <= m.hi; k0 += 128) {
                            int32_t o[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int k = k0 + 32 * u;
                                o[u] = k <= m.hi ? d[k - m.base] : WF_NULL;
                            }
                            extend_n<4>(A, PR, pat, txt, k0, 32, o);
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int k = k0 + 32 * u;
                                if (k <= m.hi && o[u] != WF_NULL) d[k - m.base] = o[u];
                                // end-to-end check on the lane that holds diagonal tlen-plen
                                if (k == k_end && o[u] != WF_NULL && o[u] >= tlen) reached = true;
                            }
                        }
                    } else {
                        reached = fused_reached;
                    }
                    if (__any_sync(0xffffffffu, reached)) {
                        end_score = s;
                        break;
                    }
                } else if (num_null > A.max_score_scope) {
                    status = -3;  // end unreachable (cannot happen end-to-end without heuristics)
                    break;
                }
            }
            // ---- compute s+1
            ++s;
            if (s > smax) {
                status = WFA_OVERFLOW;
                break;
            }
            if (s % HDR_CHUNK == 0) {
                const int64_t hb = warp_alloc(A, al, (int64_t)sizeof(ScoreHdr) * HDR_CHUNK, lane);
                if (hb < 0) {
                    status = WFA_RETRY;
                    break;
                }
                if (lane == 0) ctab[s / HDR_CHUNK] = hb;
                __syncwarp();
            }
            ScoreHdr *OH = hdr_ptr(A, ctab, s);
            const CompHdr NUL{1, -1, 0, 0, 0};
            const int sm = s - P.x, so1 = s - P.o1 - P.e1, se1 = s - P.e1, so2 = s - P.o2 - P.e2, se2 = s - P.e2;
            const CompHdr m_misms = sm >= 0 ? HR.get(A, ctab, sm, s)->c[CM] : NUL;
            const CompHdr m_open1 = so1 >= 0 ? HR.get(A, ctab, so1, s)->c[CM] : NUL;
            const CompHdr i1 = se1 >= 0 ? HR.get(A, ctab, se1, s)->c[CI1] : NUL;
            const CompHdr d1 = se1 >= 0 ? HR.get(A, ctab, se1, s)->c[CD1] : NUL;
            const CompHdr m_open2 = so2 >= 0 ? HR.get(A, ctab, so2, s)->c[CM] : NUL;
            const CompHdr i2 = se2 >= 0 ? HR.get(A, ctab, se2, s)->c[CI2] : NUL;
            const CompHdr d2 = se2 >= 0 ? HR.get(A, ctab, se2, s)->c[CD2] : NUL;
            const bool n_mm = m_misms.lo > m_misms.hi, n_o1 = m_open1.lo > m_open1.hi, n_i1 = i1.lo > i1.hi,
                       n_d1 = d1.lo > d1.hi, n_o2 = m_open2.lo > m_open2.hi, n_i2 = i2.lo > i2.hi,
                       n_d2 = d2.lo > d2.hi;
            if (n_mm && n_o1 && n_i1 && n_d1 && n_o2 && n_i2 && n_d2) {
                if (lane == 0) {
                    for (int c = 0; c < 5; ++c) OH->c[c] = NUL;
                    if (HR.rs)
                        for (int c = 0; c < 5; ++c) HR.ring[s & (HR.rs - 1)].c[c] = NUL;
                }
                __syncwarp();
                ++num_null;
                fused_reached = false;
                continue;
            }
            num_null = 0;
            fused_reached = false;
            // limits (null inputs contribute lo=1, hi=-1)
            int lo = m_misms.lo, hi = m_misms.hi;
            lo = min(lo, m_open1.lo - 1), hi = max(hi, m_open1.hi + 1);
            lo = min(lo, i1.lo + 1), hi = max(hi, i1.hi + 1);
            lo = min(lo, d1.lo - 1), hi = max(hi, d1.hi - 1);
            lo = min(lo, m_open2.lo - 1), hi = max(hi, m_open2.hi + 1);
            lo = min(lo, i2.lo + 1), hi = max(hi, i2.hi + 1);
            lo = min(lo, d2.lo - 1), hi = max(hi, d2.hi - 1);
            const bool a_i1 = !n_o1 || !n_i1, a_d1 = !n_o1 || !n_d1, a_i2 = !n_o2 || !n_i2, a_d2 = !n_o2 || !n_d2;
            const int width = hi - lo + 1;
            // a wavefront wider than a warp's share: the cluster kernel re-runs the pair.  Above
            // wide_width always; above wide_width_tail once every pair has started and at most
            // wide_tail_pairs still run on warps (the batch's tail, whose idle SMs the cluster
            // kernel puts to work)
            if (!PIG && A.wide_width > 0 && width > A.wide_width_tail) {
                int drained = 0;
                if (lane == 0)
                    drained = *(volatile int32_t *)A.queue >= A.n &&
                              *(volatile int32_t *)(A.queue + 1) <= A.wide_tail_pairs;
                drained = __shfl_sync(0xffffffffu, drained, 0);
                if (width > A.wide_width || drained) {
                    status = WFA_WIDE;
                    break;
                }
            }
            CompHdr out[5];
            for (int c = 0; c < 5; ++c) out[c] = NUL;
            const bool alloc_c[5] = {true, a_i1, a_d1, a_i2, a_d2};
            if constexpr (PIG) {
                if (width > rcap) {
                    const int nc = max(2 * rcap, (width + 3) & ~3);
                    const int64_t nb = warp_alloc(A, al, ring_arrays * nc * 4, lane);
                    if (nb < 0) {
                        status = WFA_RETRY;
                        break;
                    }
                    rcap = nc, rbase = nb;
                }
                for (int c = 0; c < 5; ++c)
                    if (alloc_c[c])
                        out[c] = CompHdr{lo, hi, lo, rcap, rbase + pig_slot(c, s, SR, R1, R2) * rcap * 4};
            } else {
                const int64_t wb = (((int64_t)width * 4) + 15) & ~(int64_t)15;
                int nstore = 1;
                if (!A.singletrack) nstore += (int)a_i1 + (int)a_d1 + (int)a_i2 + (int)a_d2;
                if (A.singletrack && width > ring_cap) {
                    status = WFA_OVERFLOW;
                    break;
                }
                const int64_t blk = warp_alloc(A, al, wb * nstore, lane);
                if (blk < 0) {
                    status = WFA_RETRY;
                    break;
                }
                int64_t o = blk;
                for (int c = 0; c < 5; ++c) {
                    if (!alloc_c[c]) continue;
                    int64_t place;
                    if (c == CM || !A.singletrack) place = o, o += wb;
                    else place = ring + ((int64_t)((s % R) * 4 + (c - 1)) * ring_cap) * 4;
                    out[c] = CompHdr{lo, hi, lo, 0, place};
                }
            }
            int32_t *oM = (int32_t *)(A.pool + out[CM].off);
            int32_t *oI1 = a_i1 ? (int32_t *)(A.pool + out[CI1].off) : nullptr;
            int32_t *oD1 = a_d1 ? (int32_t *)(A.pool + out[CD1].off) : nullptr;
            int32_t *oI2 = a_i2 ? (int32_t *)(A.pool + out[CI2].off) : nullptr;
            int32_t *oD2 = a_d2 ? (int32_t *)(A.pool + out[CD2].off) : nullptr;
            // trimmed ends (wavefront/wavefront_compute.c:654-690): the lowest and highest
            // diagonal whose offset lies in the matrix, per component, from the lanes' values
            int kmin[5], kmax[5];
#pragma unroll
            for (int c = 0; c < 5; ++c) kmin[c] = INT_MAX, kmax[c] = INT_MIN;
            if constexpr (PIG) {
                // PIG_U diagonals per lane at a time (every lane runs every trip: the block
                // reservation is warp-wide)
                const CompHdr in7[7] = {m_misms, m_open1, i1, d1, m_open2, i2, d2};
                int mask = 0;
                for (int c = 0; c < 5; ++c) mask |= alloc_c[c] ? 1 << c : 0;
                for (int kb = lo; kb <= hi; kb += 32 * PIG_U) {
                    if (!pig_trip(A, PR, pat, txt, kb, lane, 32, lo, hi, in7, out, mask, rcap, al, bnext, bend, kmin, kmax,
                                  fused_reached)) {
                        status = WFA_RETRY;
                        break;
                    }
                }
                if (status != 0) break;
            } else {
                // WU diagonals per lane at a time: all input loads before any output store
                const InHdr h_mm = in_hdr(A, m_misms), h_o1 = in_hdr(A, m_open1), h_i1 = in_hdr(A, i1),
                            h_d1 = in_hdr(A, d1), h_o2 = in_hdr(A, m_open2), h_i2 = in_hdr(A, i2),
                            h_d2 = in_hdr(A, d2);
                for (int k0 = lo + lane; k0 <= hi; k0 += 32 * WU) {
                    int32_t ins1[WU], ins2[WU], del1[WU], del2[WU], misms[WU];
    #pragma unroll
                    for (int u = 0; u < WU; ++u) {
                        const int k = k0 + 32 * u;
                        ins1[u] = max(getv(h_o1, k - 1), getv(h_i1, k - 1)) + 1;
                        ins2[u] = max(getv(h_o2, k - 1), getv(h_i2, k - 1)) + 1;
                        del1[u] = max(getv(h_o1, k + 1), getv(h_d1, k + 1));
                        del2[u] = max(getv(h_o2, k + 1), getv(h_d2, k + 1));
                        misms[u] = getv(h_mm, k) + 1;
                    }
                    // the gap components are final: store them (and their trimmed ends) first, so
                    // that only M stays live across its extension
                    int32_t mo[WU];
    #pragma unroll
                    for (int u = 0; u < WU; ++u) {
                        const int k = k0 + 32 * u;
                        const int32_t best = max(max(del1[u], del2[u]), max(misms[u], max(ins1[u], ins2[u])));
                        mo[u] = (k <= hi && in_matrix(best, k, plen, tlen)) ? best : WF_NULL;
                        if (k > hi) continue;
                        if (oI1) oI1[k - lo] = ins1[u];
                        if (oD1) oD1[k - lo] = del1[u];
                        if (oI2) oI2[k - lo] = ins2[u];
                        if (oD2) oD2[k - lo] = del2[u];
                        const int32_t vals[4] = {ins1[u], del1[u], ins2[u], del2[u]};
    #pragma unroll
                        for (int c = 0; c < 4; ++c)
                            if (in_matrix(vals[c], k, plen, tlen))
                                kmin[c + 1] = min(kmin[c + 1], k), kmax[c + 1] = max(kmax[c + 1], k);
                        if (mo[u] != WF_NULL) kmin[CM] = min(kmin[CM], k), kmax[CM] = max(kmax[CM], k);
                    }
                    // then M[s], extended (the extend step of the next iteration, fused: the
                    // offsets never round-trip through memory unextended)
                    extend_n<WU>(A, PR, pat, txt, k0, 32, mo);
    #pragma unroll
                    for (int u = 0; u < WU; ++u) {
                        const int k = k0 + 32 * u;
                        if (k > hi) break;
                        if (k == k_end && mo[u] != WF_NULL && mo[u] >= tlen) fused_reached = true;
                        oM[k - lo] = mo[u];
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                if (!alloc_c[c]) continue;
                const int th = __reduce_max_sync(0xffffffffu, kmax[c]);
                const int tl = __reduce_min_sync(0xffffffffu, kmin[c]);
                // no diagonal in the matrix: the empty range [lo, lo-1] of the scan
                if (th == INT_MIN) out[c].hi = out[c].lo - 1;
                else out[c].lo = tl, out[c].hi = th;
            }
            if (lane == 0) {
                for (int c = 0; c < 5; ++c) OH->c[c] = out[c];
                if (HR.rs)
                    for (int c = 0; c < 5; ++c) HR.ring[s & (HR.rs - 1)].c[c] = out[c];
            }
            __syncwarp();
        }
        // ---- backtrace (lane 0)
        if (lane == 0) {
            finish_pair<PIG>(A, PR, idx, pat, txt, ctab, HR, status, end_score, s, al.used);
            atomicSub(A.queue + 1, 1);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------
// Cluster kernel for pairs whose wavefronts outgrow a warp (high memory: standard and
// Singletrack).  One cluster of CL CTAs (WIDE_NT threads each) per pair, one cluster barrier
// per score:
//   1. every thread of the cluster computes and extends the diagonals lo + gtid + GT*u of the
//      plan (gtid = rank * WIDE_NT + thread, GT = CL * WIDE_NT), and each warp folds its
//      trimmed ends per component, and whether the end cell was reached, into its CTA's
//      partials;
//   2. cluster barrier;
//   3. warp 0 of every CTA gathers all CTAs' partials through distributed shared memory,
//      and its lane 0 (the CTA's planner) finishes the score's headers and plans the next
//      score.  Every planner holds the same state (the headers of the last scores in a
//      shared-memory ring, the pool position), so all plans agree without being exchanged.
// Pool space is carved deterministically out of reserve chunks that thread 0 of the first
// CTA (the leader) takes from the pool one score ahead of need and announces to every CTA
// through distributed shared memory before the barrier; the leader alone writes the pool
// copy of the headers and the chunk table that the backtrace reads.  The cell arithmetic,
// the limits, the trimming and the backtrace are the warp kernel's; only the split of the
// diagonals differs, so the results are identical.  Offsets written by other CTAs are read
// through L2 (ld.global.cg), after the barrier's release/acquire.
constexpr int WIDE_NT = 384;
constexpr int WIDE_CHUNKS = 8;  // reserve chunks a planner keeps track of (a ring)

// A reserve chunk announced by the leader: for pair `tag`, the planners' chunk number `seq`
// (off < 0: the pool is exhausted).
struct WideAnn {
    int tag, seq;
    int64_t off, len;
};

// The planner's state (lane 0 of warp 0 in every CTA; identical in all of them).
struct WidePlanner {
    int pi, idx;  // queue position and pair
    int s, num_null, status, end_score, smax, R, ring_cap;
    int lo_all, hi_all;  // the union of the planned diagonal ranges so far
    int64_t ring, hdr_off, ctab_off;
    int64_t cur, end;    // carving position in the current chunk
    int nchunks, cidx;   // chunks received, chunk being carved
    bool exhausted;
};

// Reserve chunk size: large (few pool atomics), smaller in a small pool.
__device__ __forceinline__ int64_t wide_chunk(const WfaArgs &A, int64_t need) {
    const int64_t base = min((int64_t)64 << 20, max((int64_t)1 << 20, A.pool_bytes / 64));
    return ((max(base, 2 * need) + 255) & ~(int64_t)255);
}

__global__ void __launch_bounds__(WIDE_NT, 1) wfa_wide_kernel(WfaArgs A, int rs) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31;
    const int GT = CL * WIDE_NT, gtid = rank * WIDE_NT + tid;
    const bool planner = tid == 0;
    const bool leader = rank == 0 && tid == 0;
    const WfaPen P = A.pen;
    __shared__ WidePlan plan;
    __shared__ WidePart part[2];
    __shared__ WideAnn ann[2];     // reserve chunks announced before the barrier of step it (it & 1)
    __shared__ WideAnn pstart[2];  // the pair of the np-th pair start (np & 1): tag = queue position,
                                   // seq = pair, off/len = its first chunk
    __shared__ int64_t qoff[WIDE_CHUNKS], qlen[WIDE_CHUNKS];  // the planner's chunks
    extern __shared__ ScoreHdr wring[];
    const HdrRing HR{wring, rs};
    if (tid < 2) {
        part_reset(part[tid]);
        ann[tid] = WideAnn{-1, -1, -1, 0};
    }
    const CompHdr NUL{1, -1, 0, 0, 0};
    WidePlanner W{};
    int64_t used = 0;  // the leader's pool bytes for the pair
    int it = 0, np = 0;

    // ---- planner helpers (lane 0 of warp 0)
    auto carve = [&](int64_t bytes) -> int64_t {
        bytes = (bytes + 15) & ~(int64_t)15;
        while (W.cur + bytes > W.end) {
            if (W.cidx + 1 >= W.nchunks) return -1;
            ++W.cidx;
            W.cur = qoff[W.cidx % WIDE_CHUNKS];
            W.end = W.cur + qlen[W.cidx % WIDE_CHUNKS];
            if (W.cur < 0) return -1;
        }
        const int64_t r = W.cur;
        W.cur += bytes;
        return r;
    };
    // bytes the next plan may carve: one header chunk and the stored components over the
    // planned range widened by one diagonal per side
    auto need_next = [&]() -> int64_t {
        const int64_t w = (int64_t)(W.hi_all - W.lo_all) + 3;
        return (int64_t)sizeof(ScoreHdr) * HDR_CHUNK + (A.singletrack ? 1 : 5) * (w * 4 + 16) + 64;
    };
    // the next plan's carves fit: in the current chunk's tail, or in one queued chunk (a
    // carve that does not fit moves on to the next chunk)
    auto reserve_ok = [&]() -> bool {
        const int64_t need = need_next();
        bool ok = W.end - W.cur >= need;
        for (int j = W.cidx + 1; j < W.nchunks; ++j) ok |= qlen[j % WIDE_CHUNKS] >= need;
        return ok;
    };
    auto set_hdr = [&](int sc, const CompHdr (&o)[5]) {
        if (leader) {
            ScoreHdr *OH = (ScoreHdr *)(A.pool + W.hdr_off) + (sc % HDR_CHUNK);
            for (int c = 0; c < 5; ++c) OH->c[c] = o[c];
        }
        if (HR.rs)
            for (int c = 0; c < 5; ++c) HR.ring[sc & (HR.rs - 1)].c[c] = o[c];
    };
    // plans the next score with a non-null input; op = DONE with W.status set if the pair stops
    auto plan_next = [&]() {
        for (;;) {
            ++W.s;
            const int s = W.s;
            if (s > W.smax) {
                W.status = WFA_OVERFLOW;
                break;
            }
            if (s % HDR_CHUNK == 0) {
                const int64_t hb = carve((int64_t)sizeof(ScoreHdr) * HDR_CHUNK);
                if (hb < 0) {
                    W.status = WFA_RETRY;
                    break;
                }
                W.hdr_off = hb;
                if (leader) A.ctab[W.ctab_off + s / HDR_CHUNK] = hb;
            }
            CompHdr in[7];
            plan_inputs(A, A.ctab + W.ctab_off, HR, s, in);
            bool all_null = true;
            for (int j = 0; j < 7; ++j) all_null &= in[j].lo > in[j].hi;
            if (all_null) {
                const CompHdr o[5] = {NUL, NUL, NUL, NUL, NUL};
                set_hdr(s, o);
                // the top of the next step: M[s] is empty
                if (++W.num_null > A.max_score_scope) {
                    W.status = -3;
                    break;
                }
                continue;
            }
            W.num_null = 0;
            int lo, hi, mask;
            plan_limits(in, lo, hi, mask);
            W.lo_all = min(W.lo_all, lo), W.hi_all = max(W.hi_all, hi);
            const int width = hi - lo + 1;
            const int64_t wb = (((int64_t)width * 4) + 15) & ~(int64_t)15;
            const int nstore = A.singletrack ? 1 : __popc(mask);
            if (A.singletrack && width > W.ring_cap) {
                W.status = WFA_OVERFLOW;
                break;
            }
            const int64_t blk = carve(wb * nstore);
            if (blk < 0) {
                W.status = WFA_RETRY;
                break;
            }
            int64_t o = blk;
            for (int c = 0; c < 5; ++c) {
                plan.out[c] = NUL;
                if (!(mask & (1 << c))) continue;
                int64_t place;
                if (c == CM || !A.singletrack) place = o, o += wb;
                else place = W.ring + ((int64_t)((s % W.R) * 4 + (c - 1)) * W.ring_cap) * 4;
                plan.out[c] = CompHdr{lo, hi, lo, 0, place};
            }
            for (int j = 0; j < 7; ++j) plan.in[j] = in[j];
            plan.op = WOP_COMPUTE, plan.lo = lo, plan.hi = hi, plan.mask = mask;
            return;
        }
        plan.op = WOP_DONE;
    };

    for (;;) {
        // ---- pair start: the leader takes the next pair and its first chunk
        if (leader) {
            WideAnn a{A.n, -1, -1, 0};
            const int pi = atomicAdd(A.queue, 1);
            if (pi < A.n) {
                const int idx = A.order[pi];
                const WfaPairDev PR = A.pairs[idx];
                const int R = (P.e1 > P.e2 ? P.e1 : P.e2) + 1;
                const int64_t ring_b = A.singletrack ? (int64_t)R * 4 * (PR.plen + PR.tlen + 8) * 4 + 16 : 0;
                const int64_t len = wide_chunk(A, ring_b + (int64_t)sizeof(ScoreHdr) * HDR_CHUNK + 4096);
                a = WideAnn{pi, idx, pool_grab(A, len), len};
                used = a.off >= 0 ? len : 0;
            }
            for (int c = 0; c < CL; ++c) *cl.map_shared_rank(&pstart[np & 1], c) = a;
        }
        cl.sync();
        if (planner) {
            const WideAnn a = pstart[np & 1];
            if (a.tag >= A.n) {
                plan.op = WOP_EXIT;
            } else {
                const WfaPairDev PR = A.pairs[a.seq];
                W = WidePlanner{};
                W.pi = a.tag, W.idx = a.seq, W.ctab_off = PR.ctab_off;
                W.smax = PR.ctab_cap * HDR_CHUNK - 1;
                W.R = (P.e1 > P.e2 ? P.e1 : P.e2) + 1;
                W.ring_cap = PR.plen + PR.tlen + 8;
                W.end_score = -1, W.lo_all = 0, W.hi_all = 0;
                W.ring = -1;
                qoff[0] = a.off, qlen[0] = a.len;
                W.nchunks = 1, W.cidx = 0, W.cur = a.off, W.end = a.off + a.len;
                W.exhausted = a.off < 0;
                if (a.off < 0) W.status = WFA_RETRY;
                if (W.status == 0 && A.singletrack) {
                    W.ring = carve((int64_t)W.R * 4 * W.ring_cap * 4);
                    if (W.ring < 0) W.status = WFA_RETRY;
                }
                const int64_t h0 = W.status == 0 ? carve((int64_t)sizeof(ScoreHdr) * HDR_CHUNK) : -1;
                const int64_t d0 = h0 >= 0 ? carve(16) : -1;
                if (W.status == 0 && d0 < 0) W.status = WFA_RETRY;
                if (W.status == 0) {
                    // M[0] = {0} on diagonal 0, extended (every planner writes the same value)
                    const int32_t o0 = (int32_t)lcp1(A, PR, A.pat + PR.poff, A.txt + PR.toff, 0, 0);
                    W.hdr_off = h0;
                    if (leader) A.ctab[PR.ctab_off] = h0;
                    *(int32_t *)(A.pool + d0) = o0;
                    const CompHdr o[5] = {CompHdr{0, 0, 0, 0, d0}, NUL, NUL, NUL, NUL};
                    set_hdr(0, o);
                    if (PR.tlen - PR.plen == 0 && o0 >= PR.tlen) W.end_score = 0;
                }
                if (W.status != 0 || W.end_score == 0) plan.op = WOP_DONE;
                else plan_next();
            }
        }
        __syncthreads();
        ++np;
        int op = plan.op;
        if (op == WOP_EXIT) break;
        const int pidx = pstart[(np - 1) & 1].seq;
        const WfaPairDev PR = A.pairs[pidx];
        const uint8_t *pat = A.pat + PR.poff, *txt = A.txt + PR.toff;
        while (op == WOP_COMPUTE) {
            // ---- 1. this thread's diagonals of the planned score
            plan_compute<true>(A, PR, pat, txt, plan, gtid, GT, part[it & 1]);
            // the leader reserves the next plan's space ahead of need
            if (leader && !W.exhausted && W.nchunks - W.cidx < WIDE_CHUNKS - 1 && !reserve_ok()) {
                const int64_t len = wide_chunk(A, need_next());
                const int64_t off = pool_grab(A, len);
                if (off >= 0) used += len;
                const WideAnn a{W.pi, W.nchunks, off, off >= 0 ? len : 0};
                for (int c = 0; c < CL; ++c) *cl.map_shared_rank(&ann[it & 1], c) = a;
            }
            cl.sync();
            // ---- 3. gather, finish the score, plan the next one (warp 0 of every CTA)
            if (tid < 32) {
                int gmin[5], gmax[5], gr = 0;
#pragma unroll
                for (int c = 0; c < 5; ++c) gmin[c] = INT_MAX, gmax[c] = INT_MIN;
                if (lane < CL) {
                    const WidePart *rp = cl.map_shared_rank(&part[it & 1], lane);
#pragma unroll
                    for (int c = 0; c < 5; ++c) gmin[c] = rp->kmin[c], gmax[c] = rp->kmax[c];
                    gr = rp->reached;
                }
#pragma unroll
                for (int c = 0; c < 5; ++c)
                    gmin[c] = __reduce_min_sync(0xffffffffu, gmin[c]), gmax[c] = __reduce_max_sync(0xffffffffu, gmax[c]);
                gr = __any_sync(0xffffffffu, gr != 0);
                if (planner) {
                    part_reset(part[(it + 1) & 1]);
                    const WideAnn a = ann[it & 1];
                    if (a.tag == W.pi && a.seq == W.nchunks) {
                        qoff[W.nchunks % WIDE_CHUNKS] = a.off, qlen[W.nchunks % WIDE_CHUNKS] = a.len;
                        ++W.nchunks;
                        if (a.off < 0) W.exhausted = true;
                    }
                    CompHdr out[5];
                    for (int c = 0; c < 5; ++c) {
                        out[c] = plan.out[c];
                        if (!(plan.mask & (1 << c))) continue;
                        // no diagonal in the matrix: the empty range [lo, lo-1] of the scan
                        if (gmax[c] == INT_MIN) out[c].hi = out[c].lo - 1;
                        else out[c].lo = gmin[c], out[c].hi = gmax[c];
                    }
                    set_hdr(W.s, out);
                    if (gr) {
                        W.end_score = W.s;
                        plan.op = WOP_DONE;
                    } else {
                        plan_next();
                    }
                }
            }
            __syncthreads();
            ++it;
            op = plan.op;
        }
        // ---- backtrace (leader)
        if (leader)
            finish_pair<false>(A, PR, W.idx, pat, txt, A.ctab + PR.ctab_off, HR, W.status, W.end_score, W.s, used);
    }
}

}  // namespace

// Header ring size for a score scope: the smallest power of two above it, 32..128
// (shared memory of 4 warps x 128 x 120 B at most), or 0 (pool reads) beyond.
static int ring_size(int scope) {
    int rs = 32;
    while (rs <= scope && rs < 256) rs <<= 1;
    return rs <= 128 ? rs : 0;
}

template <bool PIG>
static cudaError_t launch_wfa_t(const WfaArgs &a, int ctas, cudaStream_t st) {
    const int rs = ring_size(a.max_score_scope);
    const size_t smem = (size_t)4 * rs * sizeof(ScoreHdr);
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(wfa_kernel<PIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    wfa_kernel<PIG><<<ctas, 128, smem, st>>>(a, rs);
    return cudaGetLastError();
}

cudaError_t launch_wfa(const WfaArgs &a, int ctas, cudaStream_t st) {
    return a.piggyback ? launch_wfa_t<true>(a, ctas, st) : launch_wfa_t<false>(a, ctas, st);
}

static cudaLaunchConfig_t wide_config(int ctas, int cl, size_t smem, cudaStream_t st, cudaLaunchAttribute *at) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(WIDE_NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// Header ring of the cluster kernel's planners: the smallest power of two above the score
// scope, 32..1024 (0: scope too large for the cluster kernel).
static int wide_ring_size(int scope) {
    int rs = 32;
    while (rs <= scope && rs <= 1024) rs <<= 1;
    return rs <= 1024 ? rs : 0;
}

cudaError_t launch_wfa_wide(const WfaArgs &a, int clusters, int cl, cudaStream_t st) {
    const int rs = wide_ring_size(a.max_score_scope);
    if (rs == 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)rs * sizeof(ScoreHdr);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(wfa_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = wide_config(clusters * cl, cl, smem, st, at);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, wfa_wide_kernel, a, rs);
    return e != cudaSuccess ? e : cudaGetLastError();
}

int wfa_wide_clusters(int cl, int scope) {
    const int rs = wide_ring_size(scope);
    if (rs == 0) return 0;
    const size_t smem = (size_t)rs * sizeof(ScoreHdr);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(wfa_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = wide_config(cl, cl, smem, 0, at);
    int n = 0;
    return cudaOccupancyMaxActiveClusters(&n, (void *)wfa_wide_kernel, &cfg) == cudaSuccess ? n : 0;
}

namespace {

__device__ __forceinline__ uint64_t code2(uint8_t c) {
    return c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 0u;
}

// One thread per word of 32 bases.
__global__ void wfa_pack_kernel(const uint8_t *src, int64_t nbytes, uint64_t *dst, int64_t nwords) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwords) return;
    uint64_t r = 0;
    const int64_t b0 = w * 32;
    if (b0 + 32 <= nbytes) {
        const uint4 a = *reinterpret_cast<const uint4 *>(src + b0), b = *reinterpret_cast<const uint4 *>(src + b0 + 16);
        const uint32_t wd[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 32; ++i) r |= code2((uint8_t)(wd[i >> 2] >> (8 * (i & 3)))) << (2 * i);
    } else {
        for (int i = 0; i < 32 && b0 + i < nbytes; ++i) r |= code2(src[b0 + i]) << (2 * i);
    }
    dst[w] = r;
}

// One warp per pair: packed = no byte other than A, C, G, T in the pattern and the text.
__global__ void wfa_classify_kernel(const uint8_t *pat, const uint8_t *txt, WfaPairDev *pairs, int n) {
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const WfaPairDev P = pairs[i];
    bool bad = false;
    for (int j = lane; j < P.plen && !bad; j += 32) {
        const uint8_t c = pat[P.poff + j];
        bad = !(c == 'A' || c == 'C' || c == 'G' || c == 'T');
    }
    for (int j = lane; j < P.tlen && !bad; j += 32) {
        const uint8_t c = txt[P.toff + j];
        bad = !(c == 'A' || c == 'C' || c == 'G' || c == 'T');
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) pairs[i].packed = bad ? 0 : 1;
}

}  // namespace

cudaError_t launch_wfa_pack(const uint8_t *pat, int64_t pbytes, uint64_t *ppat, const uint8_t *txt, int64_t tbytes,
                            uint64_t *ptxt, WfaPairDev *pairs, int n, cudaStream_t st) {
    const int64_t pw = (pbytes + 31) / 32 + 2, tw = (tbytes + 31) / 32 + 2;
    wfa_pack_kernel<<<(unsigned)((pw + 255) / 256), 256, 0, st>>>(pat, pbytes, ppat, pw);
    wfa_pack_kernel<<<(unsigned)((tw + 255) / 256), 256, 0, st>>>(txt, tbytes, ptxt, tw);
    if (n > 0) wfa_classify_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(pat, txt, pairs, n);
    return cudaGetLastError();
}

int wfa_occupancy(bool piggyback) {
    int nb = 0;
    const cudaError_t e =
        piggyback ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wfa_kernel<true>, 128, 4 * 32 * sizeof(ScoreHdr))
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wfa_kernel<false>, 128, 4 * 32 * sizeof(ScoreHdr));
    return e == cudaSuccess ? nb : 1;
}

}  // namespace aw
