// Allocation-free entry point: the full-matrix KSW2 strip path for one pair
// whose scratch memory (pair descriptor, work-queue counter, error flag,
// strip-boundary columns, traceback bytes) lives in a fixed device array
// compiled into this library instead of in buffers the library allocates.
//
// Who needs it: callers that must not allocate device memory at call time --
// a host process whose device memory is fully reserved by its own caching
// allocator, a latency-critical serving loop that cannot afford the implicit
// device synchronisation of cudaMalloc/cudaFree, or code that runs where
// allocation is forbidden.  Such callers pass their own device buffers for the
// inputs and outputs; this entry point calls no cudaMalloc, cudaFree or other
// allocating routine.
//
// Limits and sharing (also stated in include/anchorwave_b200.h):
//   * the scratch array is AW_NOALLOC_SCRATCH_BYTES (32 MiB) per device and stays
//     resident on every GPU that loads the library until the process exits;
//   * a pair whose traceback + boundary columns exceed it is rejected;
//   * every call shares the one array: calls whose GPU work overlaps (two
//     streams, or two host threads on one device) race on it and must be
//     serialised by the caller;
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (this loads the module), so that first call should be
//     made before any stream capture begins; the address is kept for the life of
//     the process, so the device must not be reset (cudaDeviceReset) between calls;
//   * the calling thread's deadline (aw_ksw_set_deadline) does not apply here (arming
//     it needs a device word this entry does not allocate), and the deterministic
//     stop (aw_ksw_set_stop_antidiagonal) is refused: it runs on the anti-diagonal
//     kernel, which this entry does not provide;
//   * a bounded wait between the cooperating warps that gives up (a stalled strip
//     pipeline) is reported as zdropped = 1 with no CIGAR -- the full-matrix path
//     never z-drops, so zdropped = 1 from this entry always means that failure.
#include "aw_internal.h"
#include "ksw2_exact.h"
#include "../../include/anchorwave_b200.h"

#include <mutex>

namespace aw {
namespace {

// The scratch array.  In host code `g_noalloc_scratch` is only a host-side
// stand-in for the symbol, never a usable device address: the address is
// obtained per device with cudaGetSymbolAddress and passed to the kernels.
static __device__ __align__(256) uint8_t g_noalloc_scratch[AW_NOALLOC_SCRATCH_BYTES];

constexpr size_t CTRL_BYTES = 4096;  // pair descriptor, order, queue, error, result
struct Ctrl {
    KswPair pair;
    int32_t order;
    int32_t queue;
    int32_t error;
    int32_t pad;
    KswOut out;
};
static_assert(sizeof(Ctrl) <= CTRL_BYTES, "control block too large");

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
uint8_t *g_addr[MAX_DEVICES] = {nullptr};

// Resolves (once per device, with that device current) the device address of the
// scratch array.
int scratch_address(uint8_t **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        set_error("aw_ksw_extd2_device_noalloc: no current CUDA device");
        return AW_E_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(cudaGetErrorString(e));
            return AW_E_CUDA;
        }
        g_addr[dev] = (uint8_t *)p;
    }
    *out = g_addr[dev];
    return AW_OK;
}

// Writes the pair descriptor and clears the queue counter, the error flag and
// the result record: the array keeps the previous call's contents.
__global__ void noalloc_setup_kernel(Ctrl *c, int qlen, int tlen) {
    if (threadIdx.x != 0) return;
    KswPair p;
    p.qoff = 0, p.toff = 0, p.tb_off = 0, p.bnd_off = 0, p.cig_off = 0;
    p.qlen = qlen, p.tlen = tlen;
    c->pair = p;
    c->order = 0;
    c->queue = 0;
    c->error = 0;
    KswOut o = {};
    c->out = o;
}

// Copies the result to the caller's record; a pipeline stall marks it failed.
__global__ void noalloc_finish_kernel(const Ctrl *c, KswOut *dst) {
    if (threadIdx.x != 0) return;
    KswOut o = c->out;
    if (c->error) o.zdropped = 1, o.n_cigar = 0;
    *dst = o;
}

// The result of a call that ksw_extd2 answers without DP (ksw2.h:194-199 reset).
__global__ void noalloc_reset_kernel(KswOut *dst) {
    if (threadIdx.x != 0) return;
    KswOut o;
    o.score = AW_NEG_INF, o.max = 0, o.max_q = -1, o.max_t = -1;
    o.mqe = AW_NEG_INF, o.mqe_t = -1, o.mte = AW_NEG_INF, o.mte_q = -1;
    o.n_cigar = 0, o.zdropped = 0, o.reach_end = 0, o.stopped = 0;
    *dst = o;
}

int64_t al256(int64_t v) { return (v + 255) & ~(int64_t)255; }

}  // namespace
}  // namespace aw

using namespace aw;

extern "C" int aw_ksw_extd2_device_noalloc(int qlen, const uint8_t *d_query, int tlen, const uint8_t *d_target,
                                           int8_t m, const int8_t *mat, int8_t q, int8_t e, int8_t q2, int8_t e2,
                                           int flag, aw_ksw_result_t *d_result, uint32_t *d_cigar,
                                           int cigar_capacity, void *stream) {
    static_assert(sizeof(aw_ksw_result_t) == sizeof(KswOut), "result layout");
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_result || !mat || (qlen > 0 && !d_query) || (tlen > 0 && !d_target)) {
        set_error("aw_ksw_extd2_device_noalloc: null argument");
        return AW_E_INVAL;
    }
    if (exact_stop_enabled()) {
        set_error("aw_ksw_extd2_device_noalloc: the calling thread has a deterministic stop set "
                  "(aw_ksw_set_stop_antidiagonal), which needs the anti-diagonal kernel; clear it first");
        return AW_E_UNSUPPORTED;
    }
    KswScore S;
    const int rc = full_path_params(qlen, tlen, m, mat, q, e, q2, e2, flag, &S);
    if (rc == 1) {  // answered without DP
        noalloc_reset_kernel<<<1, 32, 0, st>>>((KswOut *)d_result);
        return cudaGetLastError() == cudaSuccess ? AW_OK : AW_E_CUDA;
    }
    if (rc != AW_OK) {
        set_error("aw_ksw_extd2_device_noalloc: only the full-matrix form (w < 0, no z-drop, no Singletrack, "
                  "no approximate max / extension end, match-mismatch scores <= 0) is supported");
        return AW_E_UNSUPPORTED;
    }
    const bool cigar = !(flag & AW_EZ_SCORE_ONLY);
    const int64_t bnd_bytes = al256(4 * ksw_full_bnd_words(qlen, tlen));
    const int64_t tb_bytes = cigar ? al256(ksw_full_tb_bytes(qlen, tlen)) : 0;
    if ((int64_t)CTRL_BYTES + bnd_bytes + tb_bytes > (int64_t)AW_NOALLOC_SCRATCH_BYTES) {
        set_error("aw_ksw_extd2_device_noalloc: pair too large for the fixed scratch array "
                  "(traceback + boundary columns exceed AW_NOALLOC_SCRATCH_BYTES)");
        return AW_E_NOMEM;
    }
    if (cigar && (!d_cigar || (int64_t)cigar_capacity < (int64_t)qlen + tlen)) {
        set_error("aw_ksw_extd2_device_noalloc: d_cigar must hold qlen + tlen words");
        return AW_E_INVAL;
    }
    uint8_t *base = nullptr;
    const int arc = scratch_address(&base);
    if (arc != AW_OK) return arc;
    Ctrl *ctrl = (Ctrl *)base;
    uint32_t *bnd = (uint32_t *)(base + CTRL_BYTES);
    uint8_t *tb = base + CTRL_BYTES + bnd_bytes;

    noalloc_setup_kernel<<<1, 32, 0, st>>>(ctrl, qlen, tlen);
    if (cudaGetLastError() != cudaSuccess) {
        set_error("aw_ksw_extd2_device_noalloc: setup launch failed");
        return AW_E_CUDA;
    }
    KswFullArgs a;
    a.qcodes = d_query, a.tcodes = d_target;
    a.pairs = &ctrl->pair, a.order = &ctrl->order, a.n = 1;
    a.tb = tb, a.bnd = bnd, a.out = &ctrl->out;
    a.queue = &ctrl->queue, a.error = &ctrl->error;
    a.sc = S;
    // one pair: one group of eight warps pipelining the strips
    if (launch_ksw_full(a, flag, 8, 1, 1, st) != cudaSuccess) {
        set_error("aw_ksw_extd2_device_noalloc: DP launch failed");
        return AW_E_CUDA;
    }
    if (cigar && launch_ksw_backtrack_full(&ctrl->pair, &ctrl->order, 1, tb, &ctrl->out, d_cigar, flag, st) !=
                     cudaSuccess) {
        set_error("aw_ksw_extd2_device_noalloc: traceback launch failed");
        return AW_E_CUDA;
    }
    noalloc_finish_kernel<<<1, 32, 0, st>>>(ctrl, (KswOut *)d_result);
    if (cudaGetLastError() != cudaSuccess) {
        set_error("aw_ksw_extd2_device_noalloc: finish launch failed");
        return AW_E_CUDA;
    }
    return AW_OK;
}
