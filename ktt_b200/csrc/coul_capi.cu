// coul_capi.cu -- the C ABI of libcoulktt.so (declared in include/coulktt.h).
//
// Replaces, for the Coulomb path, what KTT's CUDA compute engine does per run: context and stream
// set-up (Source/ComputeEngine/Cuda/CudaEngine.cpp:29-60), pre-launch limit checks
// (CudaEngine.cpp:117-138), the event-bracketed launch (Source/ComputeEngine/Cuda/CudaKernel.cpp:43-70)
// and the event timing (Source/ComputeEngine/Cuda/CudaEvent.cpp:30-36).  Instead of JIT-compiling
// the kernel source with #define prefixes through NVRTC, a configuration selects one of the
// ahead-of-time compiled sm_100a variants registered by the coul_fwd_*.cu translation units.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "coul_forward.cuh"
#include "coulktt.h"
#include "coul_internal.h"

using namespace coul;

namespace {

thread_local std::string g_last_error;

std::vector<VariantEntry>& registry()
{
    static std::vector<VariantEntry> v;
    static std::once_flag once;
    std::call_once(once, [] {
        register_fwd_3d_aos(v);
        register_fwd_3d_aos_z32(v);
        register_fwd_3d_soa(v);
        register_fwd_3d_const(v);
        register_fwd_3d_precise(v);
        register_fwd_3d_soft(v);
        register_fwd_3d_soft_precise(v);
        register_fwd_3d_soft_fp64m(v);
        register_fwd_3d_soft_fp64s(v);
        register_fwd_3d_fp64(v);
        register_fwd_2d(v);
        register_fwd_split(v);
        register_fwd_queue_split(v);
        register_fwd_balanced_split(v);
    });
    return v;
}

const VariantEntry* find_variant(const VariantKey& k)
{
    for (const auto& e : registry())
        if (e.key == k)
            return &e;
    return nullptr;
}

// ---- reference kernel: KTT's directCoulombSumReference semantics (one point per thread, atoms
// from global memory, FP32 accumulation, out += V), Examples/CoulombSum3d/CoulombSum3dReference.cu:1-28.
__global__ void reference_kernel(const float4* __restrict__ atoms, int64_t n, int nx, int ny, int nz, float h,
                                 float ox, float oy, float oz, int accumulate, float* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= ny || z >= nz)
        return;
    const float gx = fmaf(static_cast<float>(x), h, ox);
    const float gy = fmaf(static_cast<float>(y), h, oy);
    const float gz = fmaf(static_cast<float>(z), h, oz);
    float e = 0.0f;
    for (int64_t j = 0; j < n; ++j) {
        const float4 a = atoms[j];
        const float dx = gx - a.x, dy = gy - a.y, dz = gz - a.z;
        e = fmaf(a.w, rsqrt_mufu(fmaf(dz, dz, fmaf(dy, dy, dx * dx))), e);
    }
    const int64_t o = (static_cast<int64_t>(z) * ny + y) * nx + x;
    out[o] = accumulate ? out[o] + e : e;
}

// FP64 evaluation of the same sum, one point per thread, for validation: grid coordinates formed
// as the tiled kernels form them (one FP32 fma), then widened; every difference, square, the square
// root and the division in FP64 (correctly rounded), accumulated in FP64.  Atoms pass through shared
// memory in tiles of kRefTile by plain loads.  No register blocking and no MUFU: independent of the
// tiled kernels' arithmetic, so it can validate them during tuning.
constexpr int kRefTile = 256;

__global__ void __launch_bounds__(256) reference_fp64_kernel(const float4* __restrict__ atoms, int64_t n, int nx,
                                                             int ny, int nz, float h, float ox, float oy, float oz,
                                                             double* __restrict__ out)
{
    __shared__ float4 tile[kRefTile];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthreads = blockDim.x * blockDim.y;
    const double gx = static_cast<double>(fmaf(static_cast<float>(x), h, ox));
    const double gy = static_cast<double>(fmaf(static_cast<float>(y), h, oy));
    const double gz = static_cast<double>(fmaf(static_cast<float>(z), h, oz));
    double e = 0.0;
    for (int64_t base = 0; base < n; base += kRefTile) {
        const int cnt = static_cast<int>(n - base < kRefTile ? n - base : kRefTile);
        __syncthreads();
        for (int j = tid; j < cnt; j += nthreads)
            tile[j] = atoms[base + j];
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            const float4 a = tile[j];
            const double dx = gx - static_cast<double>(a.x);
            const double dy = gy - static_cast<double>(a.y);
            const double dz = gz - static_cast<double>(a.z);
            e += static_cast<double>(a.w) / sqrt(dx * dx + dy * dy + dz * dz);
        }
    }
    if (x < nx && y < ny && z < nz)
        out[(static_cast<int64_t>(z) * ny + y) * nx + x] = e;
}

// (x, y, z, q) -> (x, y, (z_slice - z)^2, q): KTT's 2D convention, computed on the device
// (the iterative example does it on the host per slice: CoulombSum3dIterative.cpp:160-179).
__global__ void slice_atoms_kernel(const float4* __restrict__ in, int64_t n, float zs, float4* __restrict__ out)
{
    const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    const float4 a = in[j];
    const float dz = zs - a.z;
    out[j] = make_float4(a.x, a.y, dz * dz, a.w);
}

__global__ void pack_atoms_kernel(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                                  const float* __restrict__ q, int64_t n, float4* __restrict__ out)
{
    const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j < n)
        out[j] = make_float4(x[j], y[j], z[j], q != nullptr ? q[j] : 0.0f);
}

// Self-test of the bounded-wait machinery: one CTA arms an mbarrier for one arrival and waits on
// it with a short budget.  With arrive != 0 the arrival happens and the wait succeeds; with
// arrive == 0 nothing ever arrives, the wait expires, and the kernel records kStatusTimeout in the
// context's status word and returns -- the host then sees COUL_ERR_TIMEOUT.
__global__ void probe_wait_kernel(int arrive, uint64_t budget_ns, int* status)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0)
        mbar_arrive_expect_tx(&bar, 0);
    const bool ok = mbar_wait_bounded(&bar, 0, budget_ns);
    if (__syncthreads_or(ok ? 0 : 1) && threadIdx.x == 0)
        report_status(status, kStatusTimeout);
}

}  // namespace

// struct coul_ctx is defined in coul_internal.h (shared with the batched and adjoint units).


namespace coul {

int set_error(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_error(cudaError_t e, const char* what)
{
    return set_error(COUL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// cuCtxSetCurrent from the driver, through the runtime's entry-point query (no link to libcuda).
using CtxSetCurrentFn = int (*)(void*);

CtxSetCurrentFn ctx_set_current_fn()
{
    static CtxSetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult status{};
        if (cudaGetDriverEntryPoint("cuCtxSetCurrent", &p, cudaEnableDefault, &status) != cudaSuccess ||
            status != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<CtxSetCurrentFn>(p);
    }();
    return fn;
}

int ctx_activate(coul_ctx* ctx)
{
    if (ctx->user_context != nullptr) {
        // the caller's context, made current on this thread; the runtime calls below then use it
        const CtxSetCurrentFn set_current = ctx_set_current_fn();
        if (set_current == nullptr)
            return set_error(COUL_ERR_CUDA, "cuCtxSetCurrent is not available from the driver");
        const int r = set_current(ctx->user_context);
        if (r != 0)
            return set_error(COUL_ERR_CUDA, "cuCtxSetCurrent failed with driver error " + std::to_string(r));
        return COUL_OK;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaSetDevice");
    return COUL_OK;
}


int ctx_begin_timing(coul_ctx* ctx)
{
    cudaError_t e = cudaEventRecord(ctx->ev_start, ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaEventRecord");
    return COUL_OK;
}

int ctx_end_timing(coul_ctx* ctx)
{
    cudaError_t e = cudaEventRecord(ctx->ev_stop, ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaEventRecord");
    ctx->have_timing = true;
    return COUL_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int validate_tune(const coul_tune* t, int mode, int soa, const VariantEntry** out)
{
    if (t == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "tune is NULL");
    const int threads = t->block_x * t->block_y;
    if (t->block_x < 1 || t->block_y < 1 || threads > kMaxThreads)
        return set_error(COUL_ERR_DEVICE_LIMITS, "block " + std::to_string(t->block_x) + "x" +
                                                     std::to_string(t->block_y) + " is outside 1.." +
                                                     std::to_string(kMaxThreads) + " threads");
    if (t->atom_source != COUL_ATOMS_SHARED_TMA && t->atom_source != COUL_ATOMS_CONSTANT)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "unknown atom_source");
    if (t->precision < COUL_PREC_FP32 || t->precision > COUL_PREC_FP64_MERGE_SHARED)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "unknown precision");
    if (t->rsqrt_soft < 0 || (t->rsqrt_soft > 8 && t->rsqrt_soft < kSoftAlternate) || t->rsqrt_soft > kSoftAlternate + 7)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "rsqrt_soft must be in 0..8 or 10..17");
    if (t->split_form < 0 || t->split_form > 2)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "split_form must be 0 (cluster), 1 (queue) or 2 (balanced)");
    const int max_split = t->split_form == 2 ? kBalMaxGroups : t->split_form == 1 ? kMaxQueueSplit : kMaxSplit;
    if (t->atom_split < 0 || t->atom_split > max_split)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "atom_split must be in 0.." + std::to_string(max_split));
    const int split = t->atom_split >= 2 ? t->split_form + 1 : 0;
    if (split == 3 && threads * t->atom_split > kBalThreads)
        return set_error(COUL_ERR_DEVICE_LIMITS, "the balanced form's block (tile threads x atom groups) is limited to " +
                                                     std::to_string(kBalThreads) + " threads");
    if (split && (t->atom_source != COUL_ATOMS_SHARED_TMA || soa || t->precision != COUL_PREC_FP32))
        return set_error(COUL_ERR_UNSUPPORTED,
                         "the atom-split form streams float4 atoms through shared memory with FP32 accumulation");
    const int unroll = t->unroll <= 1 ? 1 : t->unroll;
    const VariantKey key{t->z_iterations, t->x_points, unroll, t->atom_source, soa, t->precision, t->rsqrt_soft, mode,
                         split};
    const VariantEntry* e = find_variant(key);
    if (e == nullptr) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "no compiled variant for z_iterations=%d x_points=%d unroll=%d atom_source=%d soa=%d "
                      "precision=%d rsqrt_soft=%d atom_split=%d mode=%s",
                      t->z_iterations, t->x_points, unroll, t->atom_source, soa, t->precision, t->rsqrt_soft,
                      t->atom_split, mode == kModeGrid3d ? "3d" : "2d");
        return set_error(COUL_ERR_UNSUPPORTED, buf);
    }
    if (out)
        *out = e;
    return COUL_OK;
}

int validate_grid(const coul_grid* g)
{
    if (g == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "grid is NULL");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "grid dimensions must be positive");
    if (!std::isfinite(g->spacing) || !std::isfinite(g->origin[0]) || !std::isfinite(g->origin[1]) ||
        !std::isfinite(g->origin[2]))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "grid spacing and origin must be finite");
    return COUL_OK;
}

// Device memory of the queue and balanced forms of the atom split, kept in the context and grown on
// demand: partial blocks and counters (the layout is each form's own).
struct SplitWorkspace {
    void* mem = nullptr;
    size_t bytes = 0;
    // The balanced form's counters (at the start of the memory, one per CTA) are known to be zero for
    // this many CTAs (0: unknown).  Its kernel leaves them at zero when it completes, so a following
    // launch of the same grid needs no reset; the queue form's use of the memory, a reallocation or
    // a timed-out kernel clears this.
    int64_t balanced_clean_ctas = 0;
};

// Resident blocks per SM of a persistent form's kernel for this block size and dynamic shared memory.
// The kernel's dynamic shared-memory attribute is only ever raised (never lowered, by any context
// object sharing the CUDA context), so every size launched before stays launchable.  Queried once per
// context object and kept: on the host these calls cost microseconds, which a call's event pair would
// otherwise count while the GPU waits for the launch.
static int resident_blocks(coul_ctx* ctx, const void* kernel, int threads, size_t smem, int* blocks)
{
    for (const auto& o : ctx->occupancy_cache)
        if (o.kernel == kernel && o.threads == threads && o.smem == smem) {
            *blocks = o.blocks_per_sm;
            return COUL_OK;
        }
    cudaError_t e;
    cudaFuncAttributes fa{};
    if ((e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess)
        return cuda_error(e, "kernel attributes");
    if (threads > fa.maxThreadsPerBlock)
        return set_error(COUL_ERR_DEVICE_LIMITS, "a block of " + std::to_string(threads) +
                                                     " threads exceeds this variant's launch bound of " +
                                                     std::to_string(fa.maxThreadsPerBlock));
    if (smem > static_cast<size_t>(fa.maxDynamicSharedSizeBytes) &&
        (e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem))) !=
            cudaSuccess)
        return cuda_error(e, "persistent form shared memory");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kernel, threads, smem)) != cudaSuccess)
        return cuda_error(e, "occupancy query");
    ctx->occupancy_cache.push_back(coul_ctx::Occupancy{kernel, threads, smem, *blocks});
    return COUL_OK;
}

// Grow the context's split workspace to `need` bytes (drains the stream before freeing the old one).
static int split_workspace(coul_ctx* ctx, size_t need, unsigned char** base)
{
    auto* ws = static_cast<SplitWorkspace*>(ctx->split_workspace_state);
    if (ws == nullptr) {
        ws = new SplitWorkspace();
        ctx->split_workspace_state = ws;
        ctx->cleanups.push_back([ws] {
            if (ws->mem)
                cudaFree(ws->mem);
            delete ws;
        });
    }
    if (need > ws->bytes) {
        ws->balanced_clean_ctas = 0;
        if (ws->mem) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ws->mem);
            ws->mem = nullptr;
            ws->bytes = 0;
        }
        cudaError_t e;
        if ((e = cudaMalloc(&ws->mem, need)) != cudaSuccess)
            return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("atom-split workspace: ") + cudaGetErrorString(e));
        ws->bytes = need;
    }
    *base = static_cast<unsigned char*>(ws->mem);
    return COUL_OK;
}

// The balanced form's resident grid, block (tile threads x atom groups), shared memory and zeroed
// counters (reset on the context's stream only when they are not known to be zero).  One counter
// and two partial-block slots per CTA.
int balanced_split_setup(coul_ctx* ctx, const VariantEntry* v, FwdLaunch& L, const coul_tune* t)
{
    const int groups = t->atom_split;
    const int tile_threads = t->block_x * t->block_y;
    const int threads = tile_threads * groups;
    const int64_t tiles = static_cast<int64_t>(L.grid.x) * L.grid.y * L.grid.z;
    if (tiles > 2147483647LL || L.p.n_atoms > 2147483647LL)
        return set_error(COUL_ERR_DEVICE_LIMITS, "the balanced form takes fewer than 2^31 point tiles and atoms");
    const int64_t values = static_cast<int64_t>(tile_threads) * t->z_iterations * t->x_points;
    L.block.z = static_cast<unsigned>(groups);
    L.split = groups;
    L.smem = static_cast<size_t>(kStages) * kBalStageAtoms * 16 + kStages * 8 +
             static_cast<size_t>(groups * values) * sizeof(float);
    cudaError_t e;
    int blocks_per_sm = 0;
    if (const int rc_occ = resident_blocks(ctx, v->occupancy_kernel, threads, L.smem, &blocks_per_sm))
        return rc_occ;
    if (blocks_per_sm < 1)
        return set_error(COUL_ERR_DEVICE_LIMITS, "the balanced form's block does not fit on an SM");
    // every CTA resident, at least one unit each
    const int64_t units = tiles * L.p.n_atoms;
    int64_t ctas = static_cast<int64_t>(blocks_per_sm) * ctx->sm_count;
    const int64_t cap = units > 0 ? units : tiles;
    if (ctas > cap)
        ctas = cap;
    // the counters first, so that their place depends on the grid alone
    const size_t done_bytes = static_cast<size_t>(ctas) * sizeof(unsigned);
    const size_t partial_offset = (done_bytes + 255) / 256 * 256;
    const size_t need = partial_offset + static_cast<size_t>(2 * ctas * values) * sizeof(float);
    unsigned char* base = nullptr;
    const int rc = split_workspace(ctx, need, &base);
    if (rc != COUL_OK)
        return rc;
    auto* ws = static_cast<SplitWorkspace*>(ctx->split_workspace_state);
    if (ws->balanced_clean_ctas != ctas) {
        if ((e = cudaMemsetAsync(base, 0, done_bytes, ctx->stream)) != cudaSuccess)
            return cuda_error(e, "balanced form counters reset");
        ws->balanced_clean_ctas = ctas;
    }
    L.queue.partial = reinterpret_cast<float*>(base + partial_offset);
    L.queue.tile_done = reinterpret_cast<unsigned*>(base);
    L.queue.counter = nullptr;
    L.queue.chunks = 2;
    L.queue.ctas = static_cast<int>(ctas);
    return COUL_OK;
}

// The queue form's persistent grid and zeroed counters, enqueued on the context's stream.
int queue_split_setup(coul_ctx* ctx, const VariantEntry* v, FwdLaunch& L, const coul_tune* t)
{
    const int threads = t->block_x * t->block_y;
    const int64_t tiles = static_cast<int64_t>(L.grid.x) * L.grid.y * L.grid.z;
    const int64_t values = static_cast<int64_t>(threads) * t->z_iterations * t->x_points;
    const size_t partial_bytes = static_cast<size_t>(tiles * t->atom_split * values) * sizeof(float);
    const size_t done_offset = (partial_bytes + 255) / 256 * 256;
    const size_t counter_offset = (done_offset + static_cast<size_t>(tiles) * sizeof(unsigned) + 255) / 256 * 256;
    const size_t need = counter_offset + 256;
    unsigned char* base = nullptr;
    const int rc = split_workspace(ctx, need, &base);
    if (rc != COUL_OK)
        return rc;
    static_cast<SplitWorkspace*>(ctx->split_workspace_state)->balanced_clean_ctas = 0;
    cudaError_t e;
    // the per-tile counters and the queue head start every launch at zero
    if ((e = cudaMemsetAsync(base + done_offset, 0, need - done_offset, ctx->stream)) != cudaSuccess)
        return cuda_error(e, "queue counters reset");
    int blocks_per_sm = 0;
    if (const int rc_occ = resident_blocks(ctx, v->occupancy_kernel, threads, L.smem, &blocks_per_sm))
        return rc_occ;
    if (blocks_per_sm < 1)
        return set_error(COUL_ERR_DEVICE_LIMITS, "the queue form's block does not fit on an SM");
    L.queue.partial = reinterpret_cast<float*>(base);
    L.queue.tile_done = reinterpret_cast<unsigned*>(base + done_offset);
    L.queue.counter = reinterpret_cast<unsigned long long*>(base + counter_offset);
    L.queue.chunks = t->atom_split;
    const int64_t items = tiles * t->atom_split;
    const int64_t ctas = static_cast<int64_t>(blocks_per_sm) * ctx->sm_count;
    L.queue.ctas = static_cast<int>(ctas < items ? ctas : items);
    return COUL_OK;
}

// Launch one forward variant over a grid; shared by the 3D AoS/SoA and 2D entry points and by
// the batched path's plain-launch baseline.
int launch_forward(coul_ctx* ctx, const VariantEntry* v, const FwdParams& prm, int mode, const coul_tune* t)
{
    FwdLaunch L{};
    L.p = prm;
    L.p.status = ctx->d_status;
    L.block = dim3(static_cast<unsigned>(t->block_x), static_cast<unsigned>(t->block_y), 1);
    const int64_t bx = static_cast<int64_t>(t->block_x) * t->x_points;
    const int64_t gx = (prm.nx + bx - 1) / bx;
    int64_t gy, gz;
    if (mode == kModeGrid3d) {
        gy = (prm.ny + t->block_y - 1) / t->block_y;
        gz = (prm.nz - prm.z_base + t->z_iterations - 1) / t->z_iterations;
    } else {
        const int64_t by = static_cast<int64_t>(t->block_y) * t->z_iterations;
        gy = (prm.ny + by - 1) / by;
        gz = 1;
    }
    if (gx > 2147483647LL || gy > 65535 || gz > 65535)
        return set_error(COUL_ERR_DEVICE_LIMITS, "grid too large for one launch");
    L.grid = dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy), static_cast<unsigned>(gz));
    L.smem = (t->atom_source == COUL_ATOMS_SHARED_TMA) ? (kStages * kTileAtoms * 16 + kStages * 8) : 0;
    if (t->precision == COUL_PREC_FP64_MERGE_SHARED)
        L.smem += shared_sums_bytes(t->block_x * t->block_y, t->z_iterations * t->x_points);
    if (v->key.split == 1) {
        L.split = t->atom_split;
        L.smem = split_smem_bytes(t->block_x * t->block_y, t->z_iterations * t->x_points);
        if (static_cast<int64_t>(L.grid.x) * L.split > 2147483647LL)
            return set_error(COUL_ERR_DEVICE_LIMITS, "grid too large for one launch");
    } else if (v->key.split == 2) {
        L.split = t->atom_split;
        const int rc = queue_split_setup(ctx, v, L, t);
        if (rc != COUL_OK)
            return rc;
    } else if (v->key.split == 3) {
        const int rc = balanced_split_setup(ctx, v, L, t);
        if (rc != COUL_OK)
            return rc;
    }
    const int xp = t->x_points;
    L.vec_store = (xp > 1 && prm.nx % xp == 0 &&
                   (reinterpret_cast<uintptr_t>(prm.out) % (sizeof(float) * (xp >= 4 ? 4 : xp))) == 0)
                      ? 1
                      : 0;
    cudaError_t e = v->launch(L, ctx->stream);
    if (e == cudaErrorLaunchOutOfResources)
        return set_error(COUL_ERR_DEVICE_LIMITS, std::string("forward launch: ") + cudaGetErrorString(e));
    if (e != cudaSuccess)
        return cuda_error(e, "forward launch");
    return COUL_OK;
}

}  // namespace coul

extern "C" {

COUL_API const char* coul_last_error(void) { return g_last_error.c_str(); }

COUL_API const char* coul_status_string(int status)
{
    switch (status) {
    case COUL_OK: return "ok";
    case COUL_ERR_INVALID_ARGUMENT: return "invalid argument";
    case COUL_ERR_CUDA: return "CUDA error";
    case COUL_ERR_UNSUPPORTED: return "unsupported configuration";
    case COUL_ERR_DEVICE_LIMITS: return "device limits exceeded";
    case COUL_ERR_TIMEOUT: return "device-side wait timed out";
    case COUL_ERR_NO_DEVICE: return "no suitable device";
    case COUL_ERR_OUT_OF_MEMORY: return "out of memory";
    default: return "unknown status";
    }
}

namespace {

// Device check and per-context resources, with the context's CUDA context already current.
int ctx_init(coul_ctx* ctx, int device)
{
    cudaDeviceProp prop{};
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaGetDeviceProperties");
    if (prop.major != 10 || prop.minor != 0)
        return set_error(COUL_ERR_NO_DEVICE, std::string("libcoulktt is built for sm_100a only; device is ") +
                                                 prop.name + " (sm_" + std::to_string(prop.major) +
                                                 std::to_string(prop.minor) + ")");
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev_start)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev_stop)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_status, sizeof(int))) != cudaSuccess ||
        (e = cudaMemset(ctx->d_status, 0, sizeof(int))) != cudaSuccess)
        return cuda_error(e, "context set-up");
    if (ctx->stream == nullptr)
        ctx->stream = ctx->own_stream;
    (void)registry();
    return COUL_OK;
}

}  // namespace

COUL_API int coul_ctx_create(int device, coul_ctx** out)
{
    if (out == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx output pointer is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return set_error(COUL_ERR_NO_DEVICE, std::string("no CUDA device: ") +
                                                 (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
    if (device < 0 || device >= count)
        return set_error(COUL_ERR_NO_DEVICE, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaSetDevice");
    auto* ctx = new coul_ctx();
    const int rc = ctx_init(ctx, device);
    if (rc) {
        coul_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return COUL_OK;
}

COUL_API int coul_ctx_create_on(void* cu_context, void* stream, coul_ctx** out)
{
    if (out == nullptr || cu_context == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "NULL CUDA context or ctx output pointer");
    *out = nullptr;
    auto* ctx = new coul_ctx();
    ctx->user_context = cu_context;
    ctx->stream = static_cast<cudaStream_t>(stream);
    int rc = ctx_activate(ctx);
    int device = -1;
    if (rc == COUL_OK) {
        const cudaError_t e = cudaGetDevice(&device);  // the device of the current (the caller's) context
        if (e != cudaSuccess)
            rc = cuda_error(e, "cudaGetDevice");
    }
    if (rc == COUL_OK)
        rc = ctx_init(ctx, device);
    if (rc) {
        if (device < 0)
            ctx->user_context = nullptr;  // nothing was created in it
        coul_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return COUL_OK;
}

COUL_API int coul_ctx_destroy(coul_ctx* ctx)
{
    if (ctx == nullptr)
        return COUL_OK;
    ctx_activate(ctx);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    orphan_batches(ctx);
    if (ctx->d_atoms_cache)
        cudaFree(ctx->d_atoms_cache);
    if (ctx->d_out_cache)
        cudaFree(ctx->d_out_cache);
    if (ctx->d_status)
        cudaFree(ctx->d_status);
    if (ctx->ev_start)
        cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop)
        cudaEventDestroy(ctx->ev_stop);
    if (ctx->own_stream)
        cudaStreamDestroy(ctx->own_stream);
    for (auto& f : ctx->cleanups)
        f();
    delete ctx;
    return COUL_OK;
}

COUL_API int coul_ctx_set_stream(coul_ctx* ctx, void* stream)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->stream = static_cast<cudaStream_t>(stream);
    return COUL_OK;
}

COUL_API void* coul_ctx_get_stream(coul_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

COUL_API void* coul_ctx_own_stream(coul_ctx* ctx) { return ctx ? static_cast<void*>(ctx->own_stream) : nullptr; }

COUL_API int coul_ctx_device(coul_ctx* ctx, int* device)
{
    if (ctx == nullptr || device == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx or device is NULL");
    *device = ctx->device;
    return COUL_OK;
}

COUL_API int coul_ctx_device_info(coul_ctx* ctx, int* sm_count, int* cc_major, int* cc_minor)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (sm_count)
        *sm_count = ctx->sm_count;
    if (cc_major)
        *cc_major = ctx->cc_major;
    if (cc_minor)
        *cc_minor = ctx->cc_minor;
    return COUL_OK;
}

COUL_API int coul_device_count(int* count)
{
    if (count == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "count is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();  // no driver or no device: report zero devices
        n = 0;
    }
    *count = n;
    return COUL_OK;
}

COUL_API int coul_device_query(int device, coul_device_props* props)
{
    if (props == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "props is NULL");
    int n = 0;
    coul_device_count(&n);
    if (device < 0 || device >= n)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "no CUDA device with index " + std::to_string(device));
    cudaDeviceProp p{};
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaGetDeviceProperties");
    std::memset(props, 0, sizeof(*props));
    std::snprintf(props->name, sizeof(props->name), "%s", p.name);
    props->global_memory = static_cast<uint64_t>(p.totalGlobalMem);
    props->shared_memory_block = static_cast<uint64_t>(p.sharedMemPerBlock);
    props->constant_memory = static_cast<uint64_t>(p.totalConstMem);
    props->max_threads_block = p.maxThreadsPerBlock;
    props->sm_count = p.multiProcessorCount;
    props->cc_major = p.major;
    props->cc_minor = p.minor;
    if ((e = cudaDriverGetVersion(&props->driver_version)) != cudaSuccess)
        return cuda_error(e, "cudaDriverGetVersion");
    return COUL_OK;
}

COUL_API int coul_synchronize(coul_ctx* ctx)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaStreamSynchronize");
    int status = 0;
    e = cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_error(e, "status read-back");
    if (status != kStatusOk) {
        cudaMemset(ctx->d_status, 0, sizeof(int));
        if (ctx->split_workspace_state)  // a kernel that gave up may have left counters behind
            static_cast<SplitWorkspace*>(ctx->split_workspace_state)->balanced_clean_ctas = 0;
        return set_error(COUL_ERR_TIMEOUT, "a kernel gave up on a bounded wait (status " + std::to_string(status) +
                                               "); its output is invalid");
    }
    return COUL_OK;
}

COUL_API int coul_elapsed_ms(coul_ctx* ctx, double* ms)
{
    if (ctx == nullptr || ms == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx or ms is NULL");
    if (!ctx->have_timing)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "no timed call yet");
    cudaError_t e = cudaEventSynchronize(ctx->ev_stop);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaEventSynchronize");
    float f = 0.0f;
    e = cudaEventElapsedTime(&f, ctx->ev_start, ctx->ev_stop);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaEventElapsedTime");
    *ms = static_cast<double>(f);
    return COUL_OK;
}

COUL_API void coul_tune_default(coul_tune* t)
{
    if (t == nullptr)
        return;
    t->block_x = 32;
    t->block_y = 4;
    t->z_iterations = 16;
    t->x_points = 4;
    t->unroll = 1;
    t->atom_source = COUL_ATOMS_SHARED_TMA;
    t->precision = COUL_PREC_FP32;
    t->rsqrt_soft = 0;
    t->atom_split = 0;
    t->split_form = 0;
}

COUL_API int coul_tune_supported(const coul_tune* t) { return validate_tune(t, kModeGrid3d, 0, nullptr); }

COUL_API int coul_tune_supported_2d(const coul_tune* t) { return validate_tune(t, kModeSlice2d, 0, nullptr); }

COUL_API int coul_variant_count(void) { return static_cast<int>(registry().size()); }

COUL_API int coul_variant_get(int i, coul_tune* t, int* is_2d, int* is_soa)
{
    if (t == nullptr || i < 0 || i >= static_cast<int>(registry().size()))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "variant index out of range");
    const VariantKey& k = registry()[static_cast<size_t>(i)].key;
    coul_tune_default(t);
    t->z_iterations = k.zi;
    t->x_points = k.xp;
    t->unroll = k.unroll;
    t->atom_source = k.src;
    t->precision = k.prec;
    t->rsqrt_soft = k.soft;
    t->atom_split = k.split ? 2 : 0;
    t->split_form = k.split ? k.split - 1 : 0;
    if (is_2d)
        *is_2d = k.mode == kModeSlice2d ? 1 : 0;
    if (is_soa)
        *is_soa = k.soa;
    return COUL_OK;
}

static int forward_3d_common(coul_ctx* ctx, const float* d_atoms, const float* d_x, const float* d_y,
                             const float* d_z, const float* d_q, int soa, int64_t n_atoms, const coul_grid* grid,
                             int z_begin, int z_end, const coul_tune* tune, int accumulate, float* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = validate_grid(grid);
    if (rc)
        return rc;
    if (z_end < 0)
        z_end = grid->nz;
    if (z_begin < 0 || z_begin >= z_end || z_end > grid->nz)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "slab [z_begin, z_end) must be a non-empty range inside the grid");
    const VariantEntry* v = nullptr;
    if ((rc = validate_tune(tune, kModeGrid3d, soa, &v)))
        return rc;
    if (n_atoms < 0)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "negative atom count");
    if (d_out == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "output pointer is NULL");
    if (n_atoms > 0) {
        if (!soa && (d_atoms == nullptr || !aligned16(d_atoms)))
            return set_error(COUL_ERR_INVALID_ARGUMENT, "atoms must be a non-NULL, 16-byte aligned float4 array");
        if (soa && (!d_x || !d_y || !d_z || !d_q || !aligned16(d_x) || !aligned16(d_y) || !aligned16(d_z) ||
                    !aligned16(d_q)))
            return set_error(COUL_ERR_INVALID_ARGUMENT, "SoA atom arrays must be non-NULL and 16-byte aligned");
    }
    if ((rc = ctx_activate(ctx)))
        return rc;
    FwdParams p{};
    p.atoms = reinterpret_cast<const float4*>(d_atoms);
    p.sx = d_x;
    p.sy = d_y;
    p.sz = d_z;
    p.sq = d_q;
    p.n_atoms = n_atoms;
    p.nx = grid->nx;
    p.ny = grid->ny;
    p.nz = z_end;
    p.z_base = z_begin;
    p.h = grid->spacing;
    p.ox = grid->origin[0];
    p.oy = grid->origin[1];
    p.oz = grid->origin[2];
    p.out = d_out;
    p.accumulate = accumulate ? 1 : 0;
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    if ((rc = launch_forward(ctx, v, p, kModeGrid3d, tune)))
        return rc;
    return ctx_end_timing(ctx);
}

COUL_API int coul_forward_3d(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                             const coul_tune* tune, int accumulate, float* d_out)
{
    return forward_3d_common(ctx, d_atoms, nullptr, nullptr, nullptr, nullptr, 0, n_atoms, grid, 0, -1, tune,
                             accumulate, d_out);
}

COUL_API int coul_forward_3d_slab(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                                  int z_begin, int z_end, const coul_tune* tune, int accumulate, float* d_out)
{
    return forward_3d_common(ctx, d_atoms, nullptr, nullptr, nullptr, nullptr, 0, n_atoms, grid, z_begin, z_end,
                             tune, accumulate, d_out);
}

COUL_API int coul_forward_3d_soa(coul_ctx* ctx, const float* d_x, const float* d_y, const float* d_z,
                                 const float* d_q, int64_t n_atoms, const coul_grid* grid, const coul_tune* tune,
                                 int accumulate, float* d_out)
{
    if (tune && tune->atom_source != COUL_ATOMS_SHARED_TMA)
        return set_error(COUL_ERR_UNSUPPORTED, "the four-array atom layout is staged through shared memory only");
    return forward_3d_common(ctx, nullptr, d_x, d_y, d_z, d_q, 1, n_atoms, grid, 0, -1, tune, accumulate, d_out);
}

COUL_API int coul_forward_3d_reference(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, const coul_grid* grid,
                                       int accumulate, float* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = validate_grid(grid);
    if (rc)
        return rc;
    if (n_atoms < 0 || d_out == nullptr || (n_atoms > 0 && (d_atoms == nullptr || !aligned16(d_atoms))))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atoms or output");
    if (grid->nz > 65535)
        return set_error(COUL_ERR_DEVICE_LIMITS, "nz above 65535");
    if ((rc = ctx_activate(ctx)))
        return rc;
    const dim3 block(16, 16, 1);
    const dim3 g((grid->nx + 15) / 16, (grid->ny + 15) / 16, grid->nz);
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    reference_kernel<<<g, block, 0, ctx->stream>>>(reinterpret_cast<const float4*>(d_atoms), n_atoms, grid->nx,
                                                   grid->ny, grid->nz, grid->spacing, grid->origin[0],
                                                   grid->origin[1], grid->origin[2], accumulate ? 1 : 0, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_error(e, "reference launch");
    return ctx_end_timing(ctx);
}

COUL_API int coul_forward_3d_reference_fp64(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms,
                                            const coul_grid* grid, double* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = validate_grid(grid);
    if (rc)
        return rc;
    if (n_atoms < 0 || d_out == nullptr || (n_atoms > 0 && (d_atoms == nullptr || !aligned16(d_atoms))))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atoms or output");
    if (grid->nz > 65535)
        return set_error(COUL_ERR_DEVICE_LIMITS, "nz above 65535");
    if ((rc = ctx_activate(ctx)))
        return rc;
    const dim3 block(16, 16, 1);
    const dim3 g((grid->nx + 15) / 16, (grid->ny + 15) / 16, grid->nz);
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    reference_fp64_kernel<<<g, block, 0, ctx->stream>>>(reinterpret_cast<const float4*>(d_atoms), n_atoms, grid->nx,
                                                        grid->ny, grid->nz, grid->spacing, grid->origin[0],
                                                        grid->origin[1], grid->origin[2], d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_error(e, "FP64 reference launch");
    return ctx_end_timing(ctx);
}

COUL_API int coul_forward_2d(coul_ctx* ctx, const float* d_atoms, int64_t n_atoms, float spacing, int nx, int ny,
                             const coul_tune* tune, int accumulate, float* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    coul_grid g{nx, ny, 1, spacing, {0.0f, 0.0f, 0.0f}};
    int rc = validate_grid(&g);
    if (rc)
        return rc;
    const VariantEntry* v = nullptr;
    if ((rc = validate_tune(tune, kModeSlice2d, 0, &v)))
        return rc;
    if (n_atoms < 0 || d_out == nullptr || (n_atoms > 0 && (d_atoms == nullptr || !aligned16(d_atoms))))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atoms or output");
    if ((rc = ctx_activate(ctx)))
        return rc;
    FwdParams p{};
    p.atoms = reinterpret_cast<const float4*>(d_atoms);
    p.n_atoms = n_atoms;
    p.nx = nx;
    p.ny = ny;
    p.nz = 1;
    p.h = spacing;
    p.out = d_out;
    p.accumulate = accumulate ? 1 : 0;
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    if ((rc = launch_forward(ctx, v, p, kModeSlice2d, tune)))
        return rc;
    return ctx_end_timing(ctx);
}

COUL_API int coul_pack_atoms(coul_ctx* ctx, const float* d_x, const float* d_y, const float* d_z, const float* d_q,
                             int64_t n_atoms, float* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (n_atoms < 0 || (n_atoms > 0 && (!d_x || !d_y || !d_z || !d_out || !aligned16(d_out))))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atom arrays");
    if (n_atoms == 0)
        return COUL_OK;
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    const int64_t blocks = (n_atoms + 255) / 256;
    pack_atoms_kernel<<<static_cast<unsigned>(blocks), 256, 0, ctx->stream>>>(d_x, d_y, d_z, d_q, n_atoms,
                                                                               reinterpret_cast<float4*>(d_out));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? COUL_OK : cuda_error(e, "pack launch");
}

COUL_API int coul_slice_atoms(coul_ctx* ctx, const float* d_xyzq, int64_t n_atoms, float z_slice, float* d_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (n_atoms < 0 || (n_atoms > 0 && (!d_xyzq || !d_out || !aligned16(d_xyzq) || !aligned16(d_out))))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad atom arrays");
    if (n_atoms == 0)
        return COUL_OK;
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    const int64_t blocks = (n_atoms + 255) / 256;
    slice_atoms_kernel<<<static_cast<unsigned>(blocks), 256, 0, ctx->stream>>>(
        reinterpret_cast<const float4*>(d_xyzq), n_atoms, z_slice, reinterpret_cast<float4*>(d_out));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? COUL_OK : cuda_error(e, "slice launch");
}

COUL_API int coul_probe_bounded_wait(coul_ctx* ctx, int arrive, uint64_t budget_ns)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (budget_ns > 2000000000ull)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "budget above 2 s");
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    probe_wait_kernel<<<1, 32, 0, ctx->stream>>>(arrive ? 1 : 0, budget_ns, ctx->d_status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_error(e, "probe launch");
    return coul_synchronize(ctx);
}

COUL_API int coul_forward_3d_host(coul_ctx* ctx, const float* h_atoms, int64_t n_atoms, const coul_grid* grid,
                                  const coul_tune* tune, float* h_out)
{
    if (ctx == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "ctx is NULL");
    int rc = validate_grid(grid);
    if (rc)
        return rc;
    if ((rc = validate_tune(tune, kModeGrid3d, 0, nullptr)))
        return rc;
    if (n_atoms < 0 || h_out == nullptr || (n_atoms > 0 && h_atoms == nullptr))
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad host buffers");
    if ((rc = ctx_activate(ctx)))
        return rc;
    const size_t abytes = static_cast<size_t>(n_atoms) * 16;
    const size_t obytes = static_cast<size_t>(grid->nx) * grid->ny * grid->nz * sizeof(float);
    cudaError_t e;
    if (abytes > ctx->atoms_cap) {
        if (ctx->d_atoms_cache)
            cudaFree(ctx->d_atoms_cache);
        ctx->d_atoms_cache = nullptr;
        ctx->atoms_cap = 0;
        if ((e = cudaMalloc(&ctx->d_atoms_cache, abytes)) != cudaSuccess)
            return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("atom buffer: ") + cudaGetErrorString(e));
        ctx->atoms_cap = abytes;
    }
    if (obytes > ctx->out_cap) {
        if (ctx->d_out_cache)
            cudaFree(ctx->d_out_cache);
        ctx->d_out_cache = nullptr;
        ctx->out_cap = 0;
        if ((e = cudaMalloc(&ctx->d_out_cache, obytes)) != cudaSuccess)
            return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("map buffer: ") + cudaGetErrorString(e));
        ctx->out_cap = obytes;
    }
    if (abytes > 0 &&
        (e = cudaMemcpyAsync(ctx->d_atoms_cache, h_atoms, abytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cuda_error(e, "atom upload");
    if ((rc = coul_forward_3d(ctx, ctx->d_atoms_cache, n_atoms, grid, tune, 0, ctx->d_out_cache)))
        return rc;
    if ((e = cudaMemcpyAsync(h_out, ctx->d_out_cache, obytes, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return cuda_error(e, "map download");
    return coul_synchronize(ctx);
}

}  // extern "C"
