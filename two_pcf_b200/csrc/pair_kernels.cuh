// Device helpers shared by the pair-counting kernels: bulk-copy staging with
// bounded mbarrier waits, threshold binning, and privatised histograms.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "tpcf_common.h"

namespace tpcf {
namespace dev {

// ------------------------------------------------------------------ TMA ---

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk (TMA, one-dimensional) copy global -> shared completing on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: each try_wait suspends the thread for a hardware time slice;
// after `limit` unsuccessful tries the caller reports a device timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// -------------------------------------------------------------- binning ---

struct AxisK {
    const float *t;  // thresholds T[0..n] in shared memory
    int n;
    int log_binning;
    float min, inv_step, inv_log_of_base, inv_log_step;
};

// Approximate bin of the natural axis variable v (fast math); only a
// starting point for locate().
__device__ __forceinline__ int approx_bin(const AxisK &ax, float v) {
    float f = ax.log_binning ? ax.inv_log_of_base * __logf(1.0f + ax.inv_log_step * (v - ax.min))
                             : (v - ax.min) * ax.inv_step;
    f = fminf(fmaxf(f, -1.0f), (float)ax.n);
    int b = (int)floorf(f);
    return b;  // NaN becomes 0 here, which locate() corrects
}

// #{k : T[k] <= x} - 1, in [-1, n], by walking from a start bin.
__device__ __forceinline__ int locate(const AxisK &ax, float x, int b) {
    while (b < ax.n && x >= ax.t[b + 1]) ++b;
    while (b >= 0 && x < ax.t[b]) --b;
    return b;
}

// True when x is within g of a threshold bounding its bin.
__device__ __forceinline__ bool near_edge(const AxisK &ax, float x, int b, float g) {
    bool nr = false;
    if (b >= 0) nr |= (x - ax.t[b]) <= g;
    if (b < ax.n) nr |= (ax.t[b + 1] - x) <= g;
    return nr;
}

// Exact: #{k : T[k] <= x} - 1 by binary search (T non-decreasing).
__device__ __forceinline__ int locate_exact(const float *t, int n, float x) {
    int lo = 0, hi = n + 1;  // count in [lo, hi]
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (t[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

// ------------------------------------------------------------ histogram ---

// 64-bit fixed-point accumulation in two 32-bit shared words: the low word
// takes the atomic add and reports its old value; a carry (or the high part
// of a negative/large increment) goes to the high word.  Exact and
// order-independent.
__device__ __forceinline__ void acc_add(uint32_t *lo, uint32_t *hi, int i, long long q) {
    const uint32_t ql = (uint32_t)q;
    const uint32_t qh = (uint32_t)((unsigned long long)q >> 32);
    const uint32_t old = atomicAdd(&lo[i], ql);
    const uint32_t up = qh + ((old + ql) < old ? 1u : 0u);
    if (up) atomicAdd(&hi[i], up);
}

// 128-bit two's-complement accumulation in global memory: g[2i] is the low
// word, g[2i+1] the high word; v is a signed 64-bit value.  Each atomicAdd
// returns the low word just before its own add, so the carry it detects is
// exact under any interleaving.
__device__ __forceinline__ void acc_add_global(unsigned long long *g, size_t i, unsigned long long v) {
    const unsigned long long old = atomicAdd(&g[2 * i], v);
    const unsigned long long up = ((old + v) < old ? 1ull : 0ull) + ((long long)v < 0 ? ~0ull : 0ull);
    if (up) atomicAdd(&g[2 * i + 1], up);
}

}  // namespace dev
}  // namespace tpcf
