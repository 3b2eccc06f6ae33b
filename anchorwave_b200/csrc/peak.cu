// Integer-ALU peak probe: the roofline denominator for the KSW2/WFA DP kernels,
// which are bound by 32-bit integer add / min / max / logic throughput rather
// than by HBM or the tensor cores.  Each thread runs 16 independent chains of
// add -> max -> min -> xor (4 ops per chain per iteration); the device
// throughput is ops / CUDA-event time over a grid of 8 CTAs x 256 threads per SM.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int CHAINS = 16;
constexpr int ITERS = 4096;

__global__ void __launch_bounds__(256) int_peak_kernel(int32_t *sink, int seed) {
    int v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = threadIdx.x * 7 + c * 13 + seed;
    const int a = seed | 1, lo = -1000000 + seed, hi = 1000000 - seed, x = seed * 3 + 5;
#pragma unroll 1
    for (int it = 0; it < ITERS; ++it) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) {
            int t = v[c] + a;
            t = max(t, lo);
            t = min(t, hi);
            v[c] = t ^ x;
        }
    }
    int acc = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) acc += v[c];
    if (acc == 0x7fffffff) sink[0] = acc;  // never true in practice; keeps the chains live
}

// The same chains on two 16-bit fields per register (the packed cells of the KSW2 strip
// kernel), using both integer pipes as that kernel does: an add of a per-field constant
// as a multiply-add by a runtime one (FMA pipe), SIMD max (ALU pipe), a second add,
// SIMD min.  The clamps keep every field far from a carry.  Each instruction is two field
// operations.
__global__ void __launch_bounds__(256) int16x2_peak_kernel(uint32_t *sink, int seed) {
    uint32_t v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = ((threadIdx.x * 7u + c * 13u + seed) & 0x0fffu) * 0x10001u + 0x10001000u;
    const uint32_t one = seed > 0 ? 1u : 3u;  // 1 at run time, unknown to the compiler
    const uint32_t a = 0x00030003u, b = 0xfffdfffeu /* -2 in both fields, as a 32-bit add */;
    const uint32_t lo = 0x08000800u + (uint32_t)(seed & 7), hi = 0x60006000u;
#pragma unroll 1
    for (int it = 0; it < ITERS; ++it) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) {
            uint32_t t = v[c] * one + a;
            t = __vmaxs2(t, lo);
            t = t * one + b;
            v[c] = __vmins2(t, hi);
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) acc += v[c];
    if (acc == 0x7fffffffu) sink[0] = acc;  // never true in practice; keeps the chains live
}

template <class K, class T>
double probe(K kernel, double ops_per_chain_iter) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0.0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0.0;
    T *sink = nullptr;
    if (cudaMalloc(&sink, 4) != cudaSuccess) return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        kernel<<<blocks, threads>>>(sink, rep + 1);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)blocks * threads * ITERS * CHAINS * ops_per_chain_iter;
        if (rep > 0 && ms > 0.f) best = ops / (ms * 1e-3) > best ? ops / (ms * 1e-3) : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return best;
}

}  // namespace

// Field operations per second of the packed 16x2 chains (2 per instruction).
extern "C" double aw_int16x2_peak_ops(void) { return probe<decltype(&int16x2_peak_kernel), uint32_t>(int16x2_peak_kernel, 8.0); }

extern "C" double aw_int32_peak_ops(void) { return probe<decltype(&int_peak_kernel), int32_t>(int_peak_kernel, 4.0); }
