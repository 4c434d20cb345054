// coul_nbody.cu -- one leapfrog-style step of the direct N-body sum, the sibling of the Coulomb map
// that KTT tunes in Examples/Nbody (Nbody.cu:103-410 tuned kernel, NbodyReference.cu:36-75 reference).
//
// For every body i (position p_i, mass m_i, velocity v_i):
//     a_i = sum_j m_j d_ij / (|d_ij|^2 + eps^2)^(3/2),  d_ij = p_j - p_i   (j = i included: d = 0)
//     p_i' = p_i + dt v_i + damping dt^2 a_i,   v_i' = v_i + dt a_i,   w components: mass kept, 0
// The pair is the Coulomb pair with a softening term and a vector accumulator: one MUFU rsqrt and
// 12 FP32 operations (3 differences, 3 FMAs for r^2 + eps^2, 1/r^2, m/r, m/r^3, 3 FMAs into a).
// The FP32 pipe bounds it (F / 12 pairs/s), so all rsqrts stay on MUFU and the FP32 work runs as
// packed FFMA2/FMUL2/FADD2 on two bodies j per instruction.
//
// Layout: each thread owns `BP` bodies i (strided by the block size so loads and stores coalesce) in
// registers; the bodies j stream through the CTA's TMA ring of 256-body float4 stages (the forward
// kernel's ring: one elected thread issues cp.async.bulk, mbarrier expect-tx, bounded waits), each
// stage is transposed once into x/y/z/m arrays, and every thread reads the bodies (j, j + 1) as
// 8-byte shared-memory broadcasts that meet a body i, held as a splat pair, in one packed
// instruction -- so no per-pair register moves are needed to form the packed operands.  With j_split = S >= 2 a
// thread-block cluster of S CTAs shares one tile of bodies i, each CTA taking 1/S of the bodies j,
// and rank 0 adds the partial accelerations from the peers' shared memory in rank order before it
// integrates and stores (for body counts too small to fill 148 SMs one tile per CTA).
#include <cuda_runtime.h>

#include <string>

#include "coul_internal.h"

namespace coul {

namespace {

struct NbodyParams {
    const float4* pos;  // x, y, z, mass
    const float4* vel;  // x, y, z, (unused)
    float4* pos_new;
    float4* vel_new;
    int64_t n;
    float dt, damping, eps2;
    int* status;
};

constexpr int kNbodyMaxThreads = 512;
constexpr int kNbodyMaxPortableSplit = 8;
constexpr int kNbodyMaxSplit = 16;  // above 8 the B200's non-portable cluster sizes
// dynamic shared memory: the TMA ring, its barriers, the transposed stage, the split's partial sums
constexpr int kNbodySoaOffset = kStages * kTileAtoms * 16 + 16;
constexpr int kNbodyRedOffset = kNbodySoaOffset + kTileAtoms * 16;
static_assert(kStages * 8 <= 16 && kNbodySoaOffset % 16 == 0, "ring barriers fit before the transposed stage");

// the widest register blocks (8 bodies i, each with three splat positions and three pair accumulators)
// need more than the 128 registers a 512-thread block leaves per thread
constexpr int nbody_max_threads(int bp) { return bp >= 8 ? 256 : kNbodyMaxThreads; }

template <int BP, int UNR, bool SPLIT>
__global__ void __launch_bounds__(nbody_max_threads(BP), 1) nbody_kernel(const NbodyParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* tiles = smem_raw;  // TMA ring of float4 (x, y, z, m) stages
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kTileAtoms * 16);
    float* soa = reinterpret_cast<float*>(smem_raw + kNbodySoaOffset);  // x[256] y[256] z[256] m[256]
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;

    uint32_t S = 1, rank = 0;
    int tile = blockIdx.x;
    if constexpr (SPLIT) {
        S = cluster_size();
        rank = cluster_rank();
        tile = static_cast<int>(blockIdx.x / S);
    }

    // bodies i of this thread: tile * (nthreads * BP) + tid + k * nthreads, each held as a splat pair
    // (-x_i, -x_i) that meets the bodies (j, j + 1) in one packed instruction; the accumulators keep
    // the even-j and odd-j partial sums in their two lanes
    const int64_t ibase = static_cast<int64_t>(tile) * nthreads * BP + tid;
    float2 nx[BP], ny[BP], nz[BP], ax[BP], ay[BP], az[BP];
#pragma unroll
    for (int k = 0; k < BP; ++k) {
        const int64_t i = ibase + static_cast<int64_t>(k) * nthreads;
        const float4 b = i < p.n ? p.pos[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        nx[k] = splat(-b.x);
        ny[k] = splat(-b.y);
        nz[k] = splat(-b.z);
        ax[k] = ay[k] = az[k] = make_float2(0.0f, 0.0f);
    }
    const float2 eps2 = splat(p.eps2);

    // this CTA's share of the bodies j
    const int64_t chunk = (p.n + S - 1) / S;
    const int64_t jbegin = chunk * rank < p.n ? chunk * rank : p.n;
    const int64_t jcount = (p.n - jbegin) < chunk ? (p.n - jbegin) : chunk;
    const float4* src = p.pos + jbegin;
    const int64_t nst = (jcount + kTileAtoms - 1) / kTileAtoms;

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < kStages; ++s)
            mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    auto stage_count = [&](int64_t s) -> int {
        const int64_t rem = jcount - s * kTileAtoms;
        return static_cast<int>(rem < kTileAtoms ? rem : kTileAtoms);
    };
    auto issue = [&](int64_t s) {
        const int buf = static_cast<int>(s % kStages);
        const uint32_t bytes = static_cast<uint32_t>(stage_count(s)) * 16u;
        mbar_arrive_expect_tx(&full[buf], bytes);
        bulk_copy_g2s(tiles + buf * kTileAtoms * 16, src + s * kTileAtoms, bytes, &full[buf]);
    };
    if (tid == 0) {
        for (int64_t s = 0; s < nst && s < kStages; ++s)
            issue(s);
    }

    bool ok = true;
    for (int64_t s = 0; s < nst; ++s) {
        const int buf = static_cast<int>(s % kStages);
        const uint32_t parity = static_cast<uint32_t>((s / kStages) & 1);
        const bool arrived = mbar_wait_bounded(&full[buf], parity);
        if (__syncthreads_or(arrived ? 0 : 1)) {
            if (tid == 0) {
                report_status(p.status, kStatusTimeout);
                for (int64_t r = s; r < nst && r < s + kStages; ++r)
                    (void)mbar_wait_bounded(&full[r % kStages], static_cast<uint32_t>((r / kStages) & 1));
            }
            ok = false;
            break;
        }
        // Transpose the stage into four arrays (so a pair of bodies j is one 8-byte broadcast load);
        // the ragged last stage is padded with far-away massless bodies, so the loop needs no bound.
        const int cnt = stage_count(s);
        const float4* tile4 = reinterpret_cast<const float4*>(tiles + buf * kTileAtoms * 16);
        for (int j = tid; j < kTileAtoms; j += nthreads) {
            const float4 b = j < cnt ? tile4[j] : make_float4(kPadCoord, kPadCoord, kPadCoord, 0.0f);
            soa[0 * kTileAtoms + j] = b.x;
            soa[1 * kTileAtoms + j] = b.y;
            soa[2 * kTileAtoms + j] = b.z;
            soa[3 * kTileAtoms + j] = b.w;
        }
        // the TMA stage is free again: order the reads before its refill, which overlaps the math
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0 && s + kStages < nst)
            issue(s + kStages);
        const float2* sx = reinterpret_cast<const float2*>(soa);
        const float2* sy = reinterpret_cast<const float2*>(soa + kTileAtoms);
        const float2* sz = reinterpret_cast<const float2*>(soa + 2 * kTileAtoms);
        const float2* sm = reinterpret_cast<const float2*>(soa + 3 * kTileAtoms);
#pragma unroll UNR
        for (int j = 0; j < kTileAtoms / 2; ++j) {
            const float2 bx = sx[j], by = sy[j], bz = sz[j], bm = sm[j];
#pragma unroll
            for (int k = 0; k < BP; ++k) {
                const float2 dx = __fadd2_rn(bx, nx[k]);
                const float2 dy = __fadd2_rn(by, ny[k]);
                const float2 dz = __fadd2_rn(bz, nz[k]);
                const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
                const float2 inv = make_float2(rsqrt_mufu(r2.x), rsqrt_mufu(r2.y));
                const float2 f = __fmul2_rn(__fmul2_rn(bm, inv), __fmul2_rn(inv, inv));
                ax[k] = __ffma2_rn(dx, f, ax[k]);
                ay[k] = __ffma2_rn(dy, f, ay[k]);
                az[k] = __ffma2_rn(dz, f, az[k]);
            }
        }
        __syncthreads();  // the four arrays are rewritten by the next stage
    }

    float a[BP][3];
#pragma unroll
    for (int k = 0; k < BP; ++k) {
        a[k][0] = ax[k].x + ax[k].y;
        a[k][1] = ay[k].x + ay[k].y;
        a[k][2] = az[k].x + az[k].y;
    }

    if constexpr (SPLIT) {
        // partial accelerations of the cluster, added by rank 0 in rank order
        float* red = reinterpret_cast<float*>(smem_raw + kNbodyRedOffset);
#pragma unroll
        for (int k = 0; k < BP; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                red[(3 * k + c) * nthreads + tid] = a[k][c];
        cluster_sync();
        if (rank == 0) {
            for (uint32_t peer = 1; peer < S; ++peer) {
                const uint32_t base = cluster_map(red, peer);
#pragma unroll
                for (int k = 0; k < BP; ++k)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        a[k][c] += ld_cluster_f32(base + 4u * static_cast<uint32_t>((3 * k + c) * nthreads + tid));
            }
        }
        cluster_sync();  // the peers' shared memory stays valid until rank 0 has read it
        if (rank != 0)
            return;
    }
    if (!ok)
        return;

    const float dt = p.dt;
    const float half = p.damping * dt * dt;
#pragma unroll
    for (int k = 0; k < BP; ++k) {
        const int64_t i = ibase + static_cast<int64_t>(k) * nthreads;
        if (i >= p.n)
            continue;
        const float4 b = p.pos[i];
        const float4 v = p.vel[i];
        p.pos_new[i] = make_float4(fmaf(half, a[k][0], fmaf(dt, v.x, b.x)), fmaf(half, a[k][1], fmaf(dt, v.y, b.y)),
                                   fmaf(half, a[k][2], fmaf(dt, v.z, b.z)), b.w);
        p.vel_new[i] = make_float4(fmaf(dt, a[k][0], v.x), fmaf(dt, a[k][1], v.y), fmaf(dt, a[k][2], v.z), 0.0f);
    }
}

using NbodyLaunch = cudaError_t (*)(const NbodyParams&, dim3, dim3, size_t, int, cudaStream_t);

template <int BP, int UNR, bool SPLIT>
cudaError_t launch_nbody(const NbodyParams& p, dim3 grid, dim3 block, size_t smem, int split, cudaStream_t stream)
{
    auto kernel = nbody_kernel<BP, UNR, SPLIT>;
    if constexpr (!SPLIT) {
        (void)split;
        kernel<<<grid, block, smem, stream>>>(p);
        return cudaGetLastError();
    } else {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(grid.x * static_cast<unsigned>(split), grid.y, grid.z);
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(split);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (split > kNbodyMaxPortableSplit) {
            cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess)
                return e;
            int clusters = 0;
            e = cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg);
            if (e != cudaSuccess)
                return e;
            if (clusters < 1)
                return cudaErrorLaunchOutOfResources;  // no SM group can hold such a cluster of these blocks
        }
        return cudaLaunchKernelEx(&cfg, kernel, p);
    }
}

struct NbodyVariant {
    int bp, unroll;
    bool split;
    NbodyLaunch launch;
};

template <int BP, int UNR>
void add_nbody(std::vector<NbodyVariant>& v)
{
    v.push_back({BP, UNR, false, &launch_nbody<BP, UNR, false>});
    v.push_back({BP, UNR, true, &launch_nbody<BP, UNR, true>});
}

const std::vector<NbodyVariant>& nbody_variants()
{
    static const std::vector<NbodyVariant> v = [] {
        std::vector<NbodyVariant> out;
        add_nbody<1, 1>(out);
        add_nbody<1, 2>(out);
        add_nbody<1, 4>(out);
        add_nbody<2, 1>(out);
        add_nbody<2, 2>(out);
        add_nbody<2, 4>(out);
        add_nbody<4, 1>(out);
        add_nbody<4, 2>(out);
        add_nbody<4, 4>(out);
        add_nbody<8, 1>(out);
        add_nbody<8, 2>(out);
        return out;
    }();
    return v;
}

int find_nbody(const coul_nbody_tune* t, const NbodyVariant** out)
{
    if (t == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "tune is NULL");
    if (t->block_x < 32 || t->block_x > kNbodyMaxThreads || t->block_x % 32 != 0)
        return set_error(COUL_ERR_DEVICE_LIMITS, "N-body block size must be a multiple of 32 in 32.." +
                                                     std::to_string(kNbodyMaxThreads));
    if (t->j_split < 0)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "j_split must not be negative");
    if (t->j_split > kNbodyMaxSplit)  // beyond the largest cluster: no form
        return set_error(COUL_ERR_UNSUPPORTED, "j_split above " + std::to_string(kNbodyMaxSplit) + " is not supported");
    if (t->block_x > nbody_max_threads(t->bodies_per_thread))
        return set_error(COUL_ERR_DEVICE_LIMITS, "8 bodies per thread allow at most 256 threads per block");
    const int unroll = t->unroll <= 1 ? 1 : t->unroll;
    const bool split = t->j_split >= 2;
    for (const auto& e : nbody_variants()) {
        if (e.bp == t->bodies_per_thread && e.unroll == unroll && e.split == split) {
            if (out)
                *out = &e;
            return COUL_OK;
        }
    }
    return set_error(COUL_ERR_UNSUPPORTED, "no compiled N-body variant for bodies_per_thread=" +
                                               std::to_string(t->bodies_per_thread) + " unroll=" + std::to_string(unroll));
}

}  // namespace

}  // namespace coul

using namespace coul;

extern "C" {

COUL_API int coul_nbody_tune_default(coul_nbody_tune* t)
{
    if (t == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "tune is NULL");
    t->block_x = 128;
    t->bodies_per_thread = 4;
    t->unroll = 2;
    t->j_split = 0;
    return COUL_OK;
}

COUL_API int coul_nbody_tune_supported(const coul_nbody_tune* t) { return find_nbody(t, nullptr); }

COUL_API int coul_nbody_step(coul_ctx* ctx, const float* d_pos_mass, const float* d_vel, int64_t n, float dt, float damping,
                             float softening_sqr, const coul_nbody_tune* tune, float* d_pos_mass_new, float* d_vel_new)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    const NbodyVariant* v = nullptr;
    int rc = find_nbody(tune, &v);
    if (rc)
        return rc;
    if (n < 0 || (n > 0 && (!aligned16(d_pos_mass) || !aligned16(d_vel) || !aligned16(d_pos_mass_new) ||
                            !aligned16(d_vel_new) || !d_pos_mass || !d_vel || !d_pos_mass_new || !d_vel_new)))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bodies must be non-NULL, 16-byte aligned float4 arrays");
    if (d_pos_mass_new == d_pos_mass || d_vel_new == d_vel)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "the step reads all old positions: outputs must not alias inputs");
    if (!(softening_sqr > 0.0f))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "softening_sqr must be positive (the j = i term divides by it)");
    if (n == 0)
        return COUL_OK;
    if ((rc = ctx_activate(ctx)))
        return rc;
    NbodyParams p{};
    p.pos = reinterpret_cast<const float4*>(d_pos_mass);
    p.vel = reinterpret_cast<const float4*>(d_vel);
    p.pos_new = reinterpret_cast<float4*>(d_pos_mass_new);
    p.vel_new = reinterpret_cast<float4*>(d_vel_new);
    p.n = n;
    p.dt = dt;
    p.damping = damping;
    p.eps2 = softening_sqr;
    p.status = ctx->d_status;
    const int64_t per_tile = static_cast<int64_t>(tune->block_x) * tune->bodies_per_thread;
    const int64_t tiles = (n + per_tile - 1) / per_tile;
    const int split = tune->j_split >= 2 ? tune->j_split : 1;
    if (tiles * split > 2147483647LL)
        return set_error(COUL_ERR_DEVICE_LIMITS, "too many bodies for one launch");
    size_t smem = kNbodyRedOffset;
    if (split > 1)
        smem += static_cast<size_t>(tune->block_x) * 3 * tune->bodies_per_thread * sizeof(float);
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    cudaError_t e = v->launch(p, dim3(static_cast<unsigned>(tiles)), dim3(static_cast<unsigned>(tune->block_x)), smem, split,
                              ctx->stream);
    if (e == cudaErrorLaunchOutOfResources)
        return set_error(COUL_ERR_DEVICE_LIMITS, std::string("N-body launch: ") + cudaGetErrorString(e));
    if (e != cudaSuccess)
        return cuda_error(e, "N-body launch");
    return ctx_end_timing(ctx);
}

}  // extern "C"
