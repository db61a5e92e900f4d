// Roofline denominators measured on the device the engine runs on: FP32 FMA
// throughput and shared-memory atomic throughput.  The pair-count kernels are
// bound by these two pipes, not by HBM, so the bench reports its achieved
// rates against these live measurements.
#include <cuda_runtime.h>

#include "engine.h"
#include "pair_kernels.cuh"

namespace tpcf {
namespace {

__global__ void fma_peak_kernel(float *out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
          x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b);
            x1 = fmaf(x1, a, b);
            x2 = fmaf(x2, a, b);
            x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b);
            x5 = fmaf(x5, a, b);
            x6 = fmaf(x6, a, b);
            x7 = fmaf(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

__device__ __forceinline__ unsigned mix(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Returning 32-bit shared atomics at random bins of a 2500-bin histogram,
// the access pattern of the pair kernels' accumulation.
__global__ void smem_atomic_kernel(unsigned long long *out, int iters) {
    constexpr int NB = 2500;
    __shared__ unsigned h[NB];
    for (int i = threadIdx.x; i < NB; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned seed = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u;
    unsigned acc = 0;
    for (int i = 0; i < iters; ++i) acc += atomicAdd(&h[mix(seed + i) % NB], 1u);
    __syncthreads();
    unsigned long long s = acc;
    for (int i = threadIdx.x; i < NB; i += blockDim.x) s += h[i];
    atomicAdd(out, s);
}

// The pair kernels' bounded wait on a shared-memory mbarrier (count 1):
// with `arrive` thread 0 completes the phase first and the wait succeeds;
// without it nothing ever arrives and the wait gives up after `limit` tries.
// One thread reports the outcome: 0 done, 4 gave up (TPCF_E_DEVICE_TIMEOUT).
__global__ void wait_selftest_kernel(int arrive, unsigned limit, int *status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        dev::mbar_init(&bar, 1);
        dev::mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0 && arrive) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(dev::smem_u32(&bar)) : "memory");
    }
    __syncthreads();
    const bool ok = dev::mbar_wait_bounded(&bar, 0u, limit);
    if (threadIdx.x == 0) *status = ok ? 0 : 4;
}

}  // namespace

int wait_selftest(Ctx *ctx, int arrive, unsigned limit, int *device_status, Error *err) {
    DevBuf<int> st;
    if (st.alloc(1) != cudaSuccess) {
        err->status = 2;
        err->msg = "allocation failed";
        return err->status;
    }
    cudaMemsetAsync(st.p, 0xff, sizeof(int), ctx->stream);
    wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>(arrive, limit, st.p);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(device_status, st.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        err->status = 3;
        err->msg = cudaGetErrorString(e);
        return err->status;
    }
    return 0;
}

int measure_peaks(Ctx *ctx, double *fp32_tflops, double *smem_atomics_per_s, Error *err) {
    cudaStream_t st = ctx->stream;
    const int blocks = ctx->num_sms * 4, threads = 512;
    DevBuf<float> fo;
    DevBuf<unsigned long long> ao;
    if (fo.alloc((size_t)blocks * threads) != cudaSuccess || ao.alloc(1) != cudaSuccess) {
        err->status = 2;
        err->msg = "allocation failed";
        return err->status;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int it = 4000;
    double best = 0;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0, st);
        fma_peak_kernel<<<blocks, threads, 0, st>>>(fo.p, it, 0.999f, 1e-3f);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)it * blocks * threads;
        best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    *fp32_tflops = best;
    best = 0;
    const int ait = 20000, ab = ctx->num_sms * 8, at = 256;
    for (int rep = 0; rep < 2; ++rep) {
        cudaEventRecord(e0, st);
        smem_atomic_kernel<<<ab, at, 0, st>>>(ao.p, ait);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::max(best, (double)ait * ab * at / (ms * 1e-3));
    }
    *smem_atomics_per_s = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err->status = 3;
        err->msg = cudaGetErrorString(e);
        return err->status;
    }
    return 0;
}

}  // namespace tpcf
