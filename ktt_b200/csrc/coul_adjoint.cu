// coul_adjoint.cu -- gradient of a loss on the 3D map with respect to charges and positions.
//
// For V_i = sum_j q_j / |r_i - r_j| and any loss L(V) with G_i = dL/dV_i (for the weighted
// least-squares loss 0.5 sum_i w_i (V_i - T_i)^2, G_i = w_i (V_i - T_i)):
//     dL/dq_j = sum_i G_i / r_ij
//     dL/dr_j = q_j sum_i G_i (r_i - r_j) / r_ij^3
// Nothing is stored per pair: 1/r is recomputed.  KTT has no adjoint; this is the B200 form of the
// transposed sum.  Each CTA owns a tile of atoms (kAdjThreads threads x A atoms in registers) and a
// chunk of grid rows; the rows' G values stream through shared memory in 256-point segments, stored
// with the point's x coordinate as {G, G, x, x} so that one broadcast 16-byte shared load hands every
// thread both operands already paired for the packed instructions (no per-point int-to-float
// conversion, which would share the XU pipe with the rsqrts), and every thread evaluates each point
// against its atoms.  Along a
// row dy and dz are constant, so per pair the work is dx, r^2 = fma(dx, dx, dy^2 + dz^2), rsqrt,
// t = G/r, accumulate t, t3 = t/r^2, accumulate t3*dx and t3 (the y and z components are dy and dz
// times the row sum of t3): 8 FP32 operations and one MUFU rsqrt.  Row partials (FP32) go into FP64
// per-atom accumulators; each (atom tile, row chunk) writes its FP64 partials, and a second kernel
// adds the chunks in a fixed order, so the result is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "coul_internal.h"

namespace coul {

constexpr int kAdjThreads = 128;
constexpr int kAdjSegment = 256;

struct AdjParams {
    const float4* atoms;
    int64_t n_atoms;
    int nx, ny, nz;
    float h, ox, oy, oz;
    const float* grad_map;   // G, nx*ny*nz, x fastest
    double* partial;         // [chunks][n_atoms][4]: sum G/r, sum G dx/r^3, sum G dy/r^3, sum G dz/r^3
    int64_t rows_per_chunk;
    int chunks;
};

// Six CTAs per SM (at most 80 registers per thread, 24 warps): the pair loop's FMA and XU work is
// balanced 8:1, so both pipes are busy at once and only more warps hide their dependency latency
// (measured at 128^3 x 8,192 atoms: 4.87 ms with six CTAs and the point loop unrolled 4 times,
// 5.11 ms with the 96-register, four-CTA form).
template <int A>
__global__ void __launch_bounds__(kAdjThreads, 6) adjoint_kernel(const AdjParams p)
{
    __shared__ float4 s_pt[kAdjSegment];
    const int tid = threadIdx.x;
    const int64_t tile_base = static_cast<int64_t>(blockIdx.x) * kAdjThreads * A;
    float ax[A], ay[A], az[A];
#pragma unroll
    for (int k = 0; k < A; ++k) {
        const int64_t j = tile_base + tid + static_cast<int64_t>(k) * kAdjThreads;
        if (j < p.n_atoms) {
            const float4 a = p.atoms[j];
            ax[k] = a.x;
            ay[k] = a.y;
            az[k] = a.z;
        } else {
            ax[k] = ay[k] = az[k] = kPadCoord;  // far away; the result is never written
        }
    }
    // FP64 per-atom accumulators, touched once per row: kept in shared memory (component-major, so
    // a warp's accesses fall on consecutive words) rather than in 2 * 4 * A registers per thread,
    // which lets more warps share an SM to hide the pair loop's dependency latency
    __shared__ double s_acc[A * 4][kAdjThreads];
#pragma unroll
    for (int c = 0; c < A * 4; ++c)
        s_acc[c][tid] = 0.0;

    const int64_t rows = static_cast<int64_t>(p.ny) * p.nz;
    const int64_t r_begin = static_cast<int64_t>(blockIdx.y) * p.rows_per_chunk;
    const int64_t r_end = r_begin + p.rows_per_chunk < rows ? r_begin + p.rows_per_chunk : rows;
    // Atoms in lane pairs (k = 2m, 2m + 1): the per-pair FP32 work runs as packed FFMA2 / FMUL2 /
    // FADD2 instructions, two atoms per instruction, halving the issue slots the FMA pipe needs.
    constexpr int P = A / 2;
    static_assert(A % 2 == 0, "atoms per thread come in lane pairs");
    float2 nax[P];
#pragma unroll
    for (int m = 0; m < P; ++m)
        nax[m] = make_float2(-ax[2 * m], -ax[2 * m + 1]);

    for (int64_t row = r_begin; row < r_end; ++row) {
        const int y = static_cast<int>(row % p.ny);
        const int z = static_cast<int>(row / p.ny);
        const float gy = fmaf(static_cast<float>(y), p.h, p.oy);
        const float gz = fmaf(static_cast<float>(z), p.h, p.oz);
        float2 dyz2[P], sq[P], sx[P], s3[P];
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float dy0 = gy - ay[2 * m], dy1 = gy - ay[2 * m + 1];
            const float dz0 = gz - az[2 * m], dz1 = gz - az[2 * m + 1];
            dyz2[m] = make_float2(fmaf(dy0, dy0, dz0 * dz0), fmaf(dy1, dy1, dz1 * dz1));
            sq[m] = make_float2(0.0f, 0.0f);
            sx[m] = make_float2(0.0f, 0.0f);
            s3[m] = make_float2(0.0f, 0.0f);
        }
        const float* grow = p.grad_map + row * static_cast<int64_t>(p.nx);
        for (int x0 = 0; x0 < p.nx; x0 += kAdjSegment) {
            const int len = p.nx - x0 < kAdjSegment ? p.nx - x0 : kAdjSegment;
            __syncthreads();
            for (int i = tid; i < len; i += kAdjThreads) {
                const float g = grow[x0 + i];
                const float x = fmaf(static_cast<float>(x0 + i), p.h, p.ox);
                s_pt[i] = make_float4(g, g, x, x);
            }
            __syncthreads();
#pragma unroll 4
            for (int i = 0; i < len; ++i) {
                const float4 pt = s_pt[i];
                const float2 g = make_float2(pt.x, pt.y);
                const float2 gx = make_float2(pt.z, pt.w);
#pragma unroll
                for (int m = 0; m < P; ++m) {
                    const float2 dx = __fadd2_rn(gx, nax[m]);
                    const float2 r2 = __ffma2_rn(dx, dx, dyz2[m]);
                    const float2 inv = make_float2(rsqrt_mufu(r2.x), rsqrt_mufu(r2.y));
                    const float2 t = __fmul2_rn(g, inv);
                    sq[m] = __fadd2_rn(sq[m], t);
                    const float2 t3 = __fmul2_rn(t, __fmul2_rn(inv, inv));
                    sx[m] = __ffma2_rn(t3, dx, sx[m]);
                    s3[m] = __fadd2_rn(s3[m], t3);
                }
            }
        }
        // dy and dz recomputed here (same values as above) rather than held through the pair loop
#pragma unroll
        for (int m = 0; m < P; ++m) {
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const int k = 2 * m + l;
                const float vq = l ? sq[m].y : sq[m].x;
                const float vx = l ? sx[m].y : sx[m].x;
                const float v3 = l ? s3[m].y : s3[m].x;
                const float dy = gy - ay[k];
                const float dz = gz - az[k];
                s_acc[4 * k + 0][tid] += static_cast<double>(vq);
                s_acc[4 * k + 1][tid] += static_cast<double>(vx);
                s_acc[4 * k + 2][tid] += static_cast<double>(dy) * static_cast<double>(v3);
                s_acc[4 * k + 3][tid] += static_cast<double>(dz) * static_cast<double>(v3);
            }
        }
    }

#pragma unroll
    for (int k = 0; k < A; ++k) {
        const int64_t j = tile_base + tid + static_cast<int64_t>(k) * kAdjThreads;
        if (j < p.n_atoms) {
            double* dst = p.partial + (static_cast<int64_t>(blockIdx.y) * p.n_atoms + j) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                dst[c] = s_acc[4 * k + c][tid];
        }
    }
}

// dq_j = sum over chunks of the partial sum; dr_j = q_j * (sum of the three position partials);
// chunks added in index order.
__global__ void adjoint_reduce_kernel(const float4* __restrict__ atoms, const double* __restrict__ partial, int64_t n,
                                      int chunks, float* __restrict__ grad_q, float* __restrict__ grad_xyz)
{
    const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < chunks; ++c) {
        const double* src = partial + (static_cast<int64_t>(c) * n + j) * 4;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            s[k] += src[k];
    }
    const double q = static_cast<double>(atoms[j].w);
    if (grad_q)
        grad_q[j] = static_cast<float>(s[0]);
    if (grad_xyz) {
        grad_xyz[3 * j + 0] = static_cast<float>(q * s[1]);
        grad_xyz[3 * j + 1] = static_cast<float>(q * s[2]);
        grad_xyz[3 * j + 2] = static_cast<float>(q * s[3]);
    }
}

struct AdjointWorkspace {
    double* partial = nullptr;
    size_t bytes = 0;
};

}  // namespace coul

using namespace coul;

extern "C" COUL_API int coul_adjoint_3d(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                                        const float* d_grad_map, float* d_grad_q, float* d_grad_xyz)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = validate_grid(grid);
    if (rc)
        return rc;
    if (n_atoms < 0 || d_grad_map == nullptr || (n_atoms > 0 && (d_atoms == nullptr || !aligned16(d_atoms))) ||
        (d_grad_q == nullptr && d_grad_xyz == nullptr))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atoms, gradient map or outputs");
    if (n_atoms == 0)
        return COUL_OK;
    if ((rc = ctx_activate(ctx)))
        return rc;

    constexpr int A = 4;
    const int64_t tiles = (n_atoms + kAdjThreads * A - 1) / (kAdjThreads * A);
    const int64_t rows = static_cast<int64_t>(grid->ny) * grid->nz;
    // enough (tile, chunk) CTAs for ~4 waves of 6 per SM, without chunks shorter than 8 rows
    const int64_t target = static_cast<int64_t>(ctx->sm_count) * 24;
    int64_t chunks = std::max<int64_t>(1, std::min<int64_t>((target + tiles - 1) / tiles, (rows + 7) / 8));
    chunks = std::min<int64_t>(chunks, 65535);
    const int64_t rows_per_chunk = (rows + chunks - 1) / chunks;
    chunks = (rows + rows_per_chunk - 1) / rows_per_chunk;
    if (tiles > 2147483647LL)
        return set_error(COUL_ERR_DEVICE_LIMITS, "too many atoms");

    // Workspace for the FP64 partials, kept in the context and grown on demand.
    static_assert(sizeof(AdjointWorkspace) > 0, "");
    auto* ws = static_cast<AdjointWorkspace*>(ctx->adjoint_workspace);
    if (ws == nullptr) {
        ws = new AdjointWorkspace();
        ctx->adjoint_workspace = ws;
        ctx->cleanups.push_back([ws] {
            if (ws->partial)
                cudaFree(ws->partial);
            delete ws;
        });
    }
    const size_t need = static_cast<size_t>(chunks) * static_cast<size_t>(n_atoms) * 4 * sizeof(double);
    cudaError_t e;
    if (need > ws->bytes) {
        if (ws->partial) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ws->partial);
            ws->partial = nullptr;
            ws->bytes = 0;
        }
        if ((e = cudaMalloc(&ws->partial, need)) != cudaSuccess)
            return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("adjoint workspace: ") + cudaGetErrorString(e));
        ws->bytes = need;
    }

    AdjParams p{};
    p.atoms = reinterpret_cast<const float4*>(d_atoms);
    p.n_atoms = n_atoms;
    p.nx = grid->nx;
    p.ny = grid->ny;
    p.nz = grid->nz;
    p.h = grid->spacing;
    p.ox = grid->origin[0];
    p.oy = grid->origin[1];
    p.oz = grid->origin[2];
    p.grad_map = d_grad_map;
    p.partial = ws->partial;
    p.rows_per_chunk = rows_per_chunk;
    p.chunks = static_cast<int>(chunks);
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    adjoint_kernel<A><<<dim3(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks)), kAdjThreads, 0, ctx->stream>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cuda_error(e, "adjoint launch");
    adjoint_reduce_kernel<<<static_cast<unsigned>((n_atoms + 255) / 256), 256, 0, ctx->stream>>>(
        p.atoms, ws->partial, n_atoms, p.chunks, d_grad_q, d_grad_xyz);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cuda_error(e, "adjoint reduction launch");
    return ctx_end_timing(ctx);
}
