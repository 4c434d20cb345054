// coul_peaks.cu -- measured pipe rates that bound the Coulomb kernels.
//
// The pair evaluation is limited by the MUFU unit (one reciprocal square root per pair) and by
// FP32 issue (two FMA-pipe operations per pair plus the Newton iterations of the FMA-pipe rsqrt
// share).  These microkernels measure, on the device in hand and at its current clocks, the whole
// GPU's MUFU rsqrt rate, its FP32 FMA rate issued as scalar FFMA and as packed FFMA2, its FP64 FMA
// rate, and the MUFU rate left when six FMAs issue beside each rsqrt; the roofline figures the
// library reports are computed from them.  (KTT reports pipe utilisation through CUPTI counters instead,
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

// Packed FP32: each FFMA2 instruction performs two FP32 FMAs (the form the pair kernels issue).
__global__ void __launch_bounds__(256) ffma2_rate_kernel(float seed, float* sink)
{
    float2 x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        x[c] = make_float2(seed + 0.125f * c + 1e-3f * threadIdx.x, seed - 0.0625f * c);
    const float2 a = make_float2(0.999f, 0.999f), b = make_float2(1e-4f, 1e-4f);
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            x[c] = __ffma2_rn(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += x[c].x + x[c].y;
    if (s == -1.0f)
        sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) dfma_rate_kernel(double seed, float* sink)
{
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        x[c] = seed + 0.125 * c + 1e-3 * threadIdx.x;
    const double a = 0.999, b = 1e-4;
    for (int it = 0; it < kIters / 4; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += x[c];
    if (s == -1.0)
        sink[blockIdx.x] = static_cast<float>(s);
}

// MUFU rsqrts with kMixFfma independent FP32 FMAs issued beside each one: the MUFU rate this keeps
// shows what a MUFU instruction costs in issue slots (at 16 rsqrt/clk/SM and one issue slot per
// MUFU instruction, six FMAs per rsqrt would still fit the 128 thread-instructions/clk/SM).
constexpr int kMixFfma = 6;

__global__ void __launch_bounds__(256) mix_rate_kernel(float seed, float* sink)
{
    float x[kChains];
    float y[kChains][kMixFfma];
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
        x[c] = seed + 0.125f * c + 1e-3f * threadIdx.x;
#pragma unroll
        for (int k = 0; k < kMixFfma; ++k)
            y[c][k] = seed * (k + 1) + c;
    }
    const float a = 0.999f, b = 1e-4f;
    for (int it = 0; it < kIters / 2; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            x[c] = coul::rsqrt_mufu(x[c]);
#pragma unroll
            for (int k = 0; k < kMixFfma; ++k)
                y[c][k] = fmaf(y[c][k], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
        s += x[c];
#pragma unroll
        for (int k = 0; k < kMixFfma; ++k)
            s += y[c][k];
    }
    if (s == -1.0f)
        sink[blockIdx.x] = s;
}

}  // namespace

using namespace coul;

extern "C" COUL_API int coul_measure_pipe_rates_ex(coul_ctx* ctx, coul_pipe_rates* out)
{
    if (ctx == nullptr || out == nullptr)
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
    const double chains = static_cast<double>(blocks) * threads * kChains;
    double best[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // operations per launch: rsqrt, scalar FMA, packed FMA lanes (2 per FFMA2), FP64 FMA, rsqrt in the mix
    const double ops[5] = {chains * kIters, chains * kIters, 2.0 * chains * kIters, chains * (kIters / 4),
                           chains * (kIters / 2)};
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        for (int k = 0; k < 5 && e == cudaSuccess; ++k) {
            cudaEventRecord(a, ctx->stream);
            switch (k) {
            case 0: mufu_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink); break;
            case 1: ffma_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink); break;
            case 2: ffma2_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink); break;
            case 3: dfma_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5, sink); break;
            default: mix_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(1.5f, sink); break;
            }
            cudaEventRecord(b, ctx->stream);
            if ((e = cudaEventSynchronize(b)) != cudaSuccess)
                break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, b);
            best[k] = std::max(best[k], ops[k] / (ms * 1e-3));
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess)
        return cuda_error(e, "pipe-rate kernels");
    int clock_khz = 0;
    cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, ctx->device);
    out->rsqrt_per_s = best[0];
    out->ffma_per_s = best[1];
    out->ffma2_lanes_per_s = best[2];
    out->dfma_per_s = best[3];
    out->rsqrt_mix6_per_s = best[4];
    out->sm_count = ctx->sm_count;
    out->max_sm_clock_khz = clock_khz;
    return COUL_OK;
}

extern "C" COUL_API int coul_measure_pipe_rates(coul_ctx* ctx, double* rsqrt_per_s, double* ffma_per_s)
{
    if (ctx == nullptr || rsqrt_per_s == nullptr || ffma_per_s == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL argument");
    // the larger of the scalar and the packed FP32 FMA rates
    coul_pipe_rates r{};
    const int rc = coul_measure_pipe_rates_ex(ctx, &r);
    if (rc != COUL_OK)
        return rc;
    *rsqrt_per_s = r.rsqrt_per_s;
    *ffma_per_s = std::max(r.ffma_per_s, r.ffma2_lanes_per_s);
    return COUL_OK;
}
