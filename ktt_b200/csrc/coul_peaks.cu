// coul_peaks.cu -- measured pipe rates that bound the Coulomb kernels.
//
// The pair evaluation is limited by the MUFU unit (one reciprocal square root per pair) and by
// FP32 issue (two FMA-pipe operations per pair plus the Newton iterations of the FMA-pipe rsqrt
// share).  These two microkernels measure, on the device in hand and at its current clocks, the
// MUFU rsqrt rate and the FP32 FMA rate of the whole GPU; the roofline figures the library
// reports are computed from them.  (KTT reports pipe utilisation through CUPTI counters instead,
// Source/ComputeEngine/Cuda/Cupti/CuptiMetricInterface.cpp:621-660.)
#include <cuda_runtime.h>

#include <algorithm>

#include "coul_internal.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) mufu_rate_kernel(float seed, float* sink)
{
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        x[c] = seed + 0.125f * c + 1e-3f * threadIdx.x;
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            x[c] = coul::rsqrt_mufu(x[c]);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += x[c];
    if (s == -1.0f)  // never true; keeps the chains live
        sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) ffma_rate_kernel(float seed, float* sink)
{
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        x[c] = seed + 0.125f * c + 1e-3f * threadIdx.x;
    const float a = 0.999f, b = 1e-4f;
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += x[c];
    if (s == -1.0f)
        sink[blockIdx.x] = s;
}

}  // namespace

using namespace coul;

extern "C" COUL_API int coul_measure_pipe_rates(coul_ctx* ctx, double* rsqrt_per_s, double* ffma_per_s)
{
    if (ctx == nullptr || rsqrt_per_s == nullptr || ffma_per_s == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL argument");
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    const int blocks = ctx->sm_count * 8;
    const int threads = 256;
    float* sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(float) * blocks);
    if (e != cudaSuccess)
        return set_error(COUL_ERR_OUT_OF_MEMORY, "sink buffer");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best_mufu = 0.0, best_ffma = 0.0;
    const double ops = static_cast<double>(blocks) * threads * kIters * kChains;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        float ms = 0.0f;
        cudaEventRecord(a, ctx->stream);
        mufu_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink);
        cudaEventRecord(b, ctx->stream);
        if ((e = cudaEventSynchronize(b)) != cudaSuccess)
            break;
        cudaEventElapsedTime(&ms, a, b);
        best_mufu = std::max(best_mufu, ops / (ms * 1e-3));
        cudaEventRecord(a, ctx->stream);
        ffma_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink);
        cudaEventRecord(b, ctx->stream);
        if ((e = cudaEventSynchronize(b)) != cudaSuccess)
            break;
        cudaEventElapsedTime(&ms, a, b);
        best_ffma = std::max(best_ffma, ops / (ms * 1e-3));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess)
        return cuda_error(e, "pipe-rate kernels");
    *rsqrt_per_s = best_mufu;
    *ffma_per_s = best_ffma;
    return COUL_OK;
}
