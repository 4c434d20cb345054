// coul_batched.cu -- many molecules with uneven atom counts and grids in one persistent launch.
//
// KTT maps the same situation onto one launch per problem from a custom launcher (the 256 slice
// launches of Examples/CoulombSum3dIterative/CoulombSum3dIterative.cpp:146-184).  Here every tile of
// every molecule's grid is a work item; items are numbered molecule by molecule, molecules in
// decreasing order of pair count (longest-processing-time first, so the smallest items fill the
// tail).  A persistent kernel -- as many CTAs as fit on the GPU at once -- claims items from a
// device counter with one atomic add per item and runs each through the same per-tile code as the
// forward kernel, the TMA atom ring carrying over from item to item.  The counter is reset by a
// memset in the same stream before each launch; the pair (memset, launch) can be captured once into
// a CUDA graph and replayed.  The plain alternative -- one forward launch per molecule -- is kept as
// the baseline.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "coul_batched.cuh"
#include "coul_internal.h"

namespace coul {

struct BatchVariant {
    int zi, xp, unroll, prec, soft;
    const void* kernel;
};

template <int ZI, int XP, int UNR, int PREC, int SOFT>
static BatchVariant batch_variant()
{
    return BatchVariant{ZI, XP, UNR, PREC, SOFT, reinterpret_cast<const void*>(&batched_kernel<ZI, XP, UNR, PREC, SOFT>)};
}

// Tile shapes compiled for the persistent kernel (the forward kernel's best shapes on B200).
static const std::vector<BatchVariant>& batch_variants()
{
    static const std::vector<BatchVariant> v{
        batch_variant<8, 2, 2, kPrecFp32, 2>(),      batch_variant<8, 2, 1, kPrecFp32, 2>(),
        batch_variant<8, 2, 2, kPrecFp32, 0>(),      batch_variant<8, 2, 1, kPrecFp32, 0>(),
        batch_variant<4, 2, 1, kPrecFp32, 2>(),      batch_variant<4, 4, 1, kPrecFp32, 2>(),
        batch_variant<8, 4, 1, kPrecFp32, 2>(),      batch_variant<16, 1, 1, kPrecFp32, 2>(),
        batch_variant<16, 2, 1, kPrecFp32, 2>(),     batch_variant<8, 2, 1, kPrecFp64Merge, 2>(),
        batch_variant<8, 2, 1, kPrecCompensated, 2>(),
        // narrow x spans for small grids (less tile padding on 57..149-point rows)
        batch_variant<8, 1, 2, kPrecFp32, 2>(),      batch_variant<8, 1, 1, kPrecFp32, 2>(),
        batch_variant<8, 1, 2, kPrecFp32, 0>(),      batch_variant<4, 1, 2, kPrecFp32, 2>(),
        // 5/16 of the rsqrts on the FMA pipe (atoms alternating between 2 and 3 of 8 lane pairs)
        batch_variant<8, 2, 2, kPrecFp32, kSoftAlternate + 2>(),
        batch_variant<8, 2, 1, kPrecFp32, kSoftAlternate + 2>(),
        // one x-y point per thread: linear x-y tiles, padded only at the end of each plane
        batch_variant<16, 1, 2, kPrecFp32, 2>(),     batch_variant<16, 1, 1, kPrecFp32, kSoftAlternate + 2>(),
        batch_variant<16, 1, 2, kPrecFp32, kSoftAlternate + 2>(), batch_variant<8, 1, 1, kPrecFp32, kSoftAlternate + 2>(),
        batch_variant<16, 1, 1, kPrecFp64Merge, 2>(),
        // FP64 merge with the sums in shared memory (the pointwise-accurate form with fewer registers)
        batch_variant<8, 2, 1, kPrecFp64MergeShared, 2>(), batch_variant<8, 2, 2, kPrecFp64MergeShared, 2>(),
        batch_variant<16, 1, 1, kPrecFp64MergeShared, 2>(), batch_variant<4, 4, 1, kPrecFp64MergeShared, 2>(),
    };
    return v;
}

}  // namespace coul

using namespace coul;

struct coul_batch {
    coul_ctx* ctx = nullptr;
    coul_tune tune{};
    std::vector<coul_molecule> molecules;  // as given (for the separate-launch baseline)
    std::vector<int> order;                // molecule indices in work-list order
    MolDesc* d_mols = nullptr;
    unsigned long long* d_counter = nullptr;
    int64_t total_items = 0;
    double total_pairs = 0.0;
    const BatchVariant* variant = nullptr;
    int grid_ctas = 0;
    size_t smem = 0;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_accumulate = -1;
};

// Frees a batch's device resources (its context current) and leaves the handle without them.
static void batch_release_device(coul_batch* b)
{
    if (b->graph_exec)
        cudaGraphExecDestroy(b->graph_exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    if (b->capture_stream)
        cudaStreamDestroy(b->capture_stream);
    if (b->d_mols)
        cudaFree(b->d_mols);
    if (b->d_counter)
        cudaFree(b->d_counter);
    b->graph_exec = nullptr;
    b->graph = nullptr;
    b->capture_stream = nullptr;
    b->d_mols = nullptr;
    b->d_counter = nullptr;
}

static void batch_release(coul_batch* b)
{
    if (b == nullptr)
        return;
    if (b->ctx) {
        auto& live = b->ctx->batches;
        live.erase(std::remove(live.begin(), live.end(), b), live.end());
    }
    batch_release_device(b);
    delete b;
}

namespace coul {

void orphan_batches(coul_ctx* ctx)
{
    for (coul_batch* b : ctx->batches) {
        batch_release_device(b);
        b->ctx = nullptr;
    }
    ctx->batches.clear();
}

}  // namespace coul

static cudaError_t launch_batched(coul_batch* b, cudaStream_t stream, int accumulate)
{
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess)
        return e;
    BatchParams p{b->d_mols, static_cast<int>(b->order.size()), b->total_items, b->d_counter, accumulate,
                  b->ctx->d_status};
    void* args[] = {&p};
    const dim3 block(static_cast<unsigned>(b->tune.block_x), static_cast<unsigned>(b->tune.block_y), 1);
    return cudaLaunchKernel(b->variant->kernel, dim3(static_cast<unsigned>(b->grid_ctas)), block, args, b->smem, stream);
}

extern "C" {

COUL_API int coul_batch_tune_supported(const coul_tune* tune)
{
    if (tune == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "tune is NULL");
    const int threads = tune->block_x * tune->block_y;
    if (tune->block_x < 1 || tune->block_y < 1 || threads > kMaxThreads)
        return set_error(COUL_ERR_DEVICE_LIMITS, "block shape outside 1..256 threads");
    const int unroll = tune->unroll <= 1 ? 1 : tune->unroll;
    for (const auto& v : batch_variants())
        if (v.zi == tune->z_iterations && v.xp == tune->x_points && v.unroll == unroll && v.prec == tune->precision &&
            v.soft == tune->rsqrt_soft && tune->atom_source == COUL_ATOMS_SHARED_TMA)
            return COUL_OK;
    return set_error(COUL_ERR_UNSUPPORTED, "no compiled persistent variant for this tile shape");
}

COUL_API int coul_batch_create(coul_ctx* ctx, const coul_molecule* molecules, int n_molecules, const coul_tune* tune,
                               coul_batch** out)
{
    if (ctx == nullptr || out == nullptr || tune == nullptr || (n_molecules > 0 && molecules == nullptr) ||
        n_molecules < 0)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "bad batch arguments");
    *out = nullptr;
    const int threads = tune->block_x * tune->block_y;
    if (tune->block_x < 1 || tune->block_y < 1 || threads > kMaxThreads)
        return set_error(COUL_ERR_DEVICE_LIMITS, "block shape outside 1..256 threads");
    const int unroll = tune->unroll <= 1 ? 1 : tune->unroll;
    const BatchVariant* variant = nullptr;
    for (const auto& v : batch_variants())
        if (v.zi == tune->z_iterations && v.xp == tune->x_points && v.unroll == unroll && v.prec == tune->precision &&
            v.soft == tune->rsqrt_soft)
            variant = &v;
    if (variant == nullptr || tune->atom_source != COUL_ATOMS_SHARED_TMA)
        return set_error(COUL_ERR_UNSUPPORTED, "no compiled persistent variant for this tile shape");
    for (int i = 0; i < n_molecules; ++i) {
        const coul_molecule& m = molecules[i];
        int rc = validate_grid(&m.grid);
        if (rc)
            return rc;
        if (m.n_atoms < 0 || m.d_out == nullptr || (m.n_atoms > 0 && (m.d_atoms == nullptr || !aligned16(m.d_atoms))))
            return set_error(COUL_ERR_INVALID_ARGUMENT, "molecule " + std::to_string(i) + ": bad atoms or output");
        if (m.grid.nx > (1 << 24) || m.grid.ny > (1 << 24) || m.grid.nz > (1 << 24))
            return set_error(COUL_ERR_INVALID_ARGUMENT, "molecule " + std::to_string(i) + ": grid too large");
    }
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;

    auto* b = new coul_batch();
    b->ctx = ctx;
    b->tune = *tune;
    b->tune.unroll = unroll;
    b->variant = variant;
    b->molecules.assign(molecules, molecules + n_molecules);
    b->order.resize(static_cast<size_t>(n_molecules));
    std::iota(b->order.begin(), b->order.end(), 0);
    auto pairs = [&](int i) {
        const coul_molecule& m = molecules[i];
        return static_cast<double>(m.grid.nx) * m.grid.ny * m.grid.nz * static_cast<double>(m.n_atoms);
    };
    std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) { return pairs(a) > pairs(c); });

    std::vector<MolDesc> descs;
    int64_t next = 0;
    for (const int i : b->order) {
        MolDesc d{};
        d.tile_begin = next;
        next += fill_mol_desc(d, molecules[i], b->tune);
        b->total_pairs += pairs(i);
        descs.push_back(d);
    }
    b->total_items = next;

    cudaError_t e;
    int blocks_per_sm = 0;
    b->smem = kStages * kTileAtoms * 16 + kStages * 8;
    if (b->tune.precision == COUL_PREC_FP64_MERGE_SHARED)
        b->smem += shared_sums_bytes(threads, b->tune.z_iterations * b->tune.x_points);
    if (b->smem > 48u * 1024u &&
        (e = cudaFuncSetAttribute(b->variant->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(b->smem))) != cudaSuccess) {
        batch_release(b);
        return cuda_error(e, "batched kernel shared memory");
    }
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, b->variant->kernel, threads, b->smem)) !=
            cudaSuccess ||
        blocks_per_sm < 1) {
        batch_release(b);
        return e != cudaSuccess ? cuda_error(e, "occupancy query")
                                : set_error(COUL_ERR_DEVICE_LIMITS, "persistent kernel does not fit on an SM");
    }
    b->grid_ctas = blocks_per_sm * ctx->sm_count;
    if ((e = cudaMalloc(&b->d_mols, sizeof(MolDesc) * std::max<size_t>(descs.size(), 1))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_counter, sizeof(unsigned long long))) != cudaSuccess ||
        (!descs.empty() && (e = cudaMemcpy(b->d_mols, descs.data(), sizeof(MolDesc) * descs.size(),
                                           cudaMemcpyHostToDevice)) != cudaSuccess) ||
        (e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        batch_release(b);
        return set_error(COUL_ERR_OUT_OF_MEMORY, std::string("batch set-up: ") + cudaGetErrorString(e));
    }
    ctx->batches.push_back(b);
    *out = b;
    return COUL_OK;
}

COUL_API int coul_batch_destroy(coul_batch* batch)
{
    if (batch == nullptr)
        return COUL_OK;
    if (batch->ctx)
        ctx_activate(batch->ctx);
    if (batch->ctx && batch->ctx->stream)
        cudaStreamSynchronize(batch->ctx->stream);
    batch_release(batch);
    return COUL_OK;
}

COUL_API int coul_batch_info(const coul_batch* batch, int64_t* work_items, int* grid_ctas, double* total_pairs)
{
    if (batch == nullptr)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (work_items)
        *work_items = batch->total_items;
    if (grid_ctas)
        *grid_ctas = batch->grid_ctas;
    if (total_pairs)
        *total_pairs = batch->total_pairs;
    return COUL_OK;
}

COUL_API int coul_batch_run(coul_ctx* ctx, coul_batch* b, int mode, int accumulate)
{
    if (ctx == nullptr || b == nullptr || b->ctx != ctx)
        return set_error(COUL_ERR_INVALID_ARGUMENT, "batch does not belong to this context");
    int rc = ctx_activate(ctx);
    if (rc)
        return rc;
    accumulate = accumulate ? 1 : 0;
    cudaError_t e = cudaSuccess;
    if (mode == COUL_BATCH_GRAPH && (b->graph_exec == nullptr || b->graph_accumulate != accumulate)) {
        // Capture (counter reset, persistent launch) once on a private stream; replay on any stream.
        if (b->graph_exec) {
            cudaGraphExecDestroy(b->graph_exec);
            b->graph_exec = nullptr;
        }
        if (b->graph) {
            cudaGraphDestroy(b->graph);
            b->graph = nullptr;
        }
        if ((e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_error(e, "graph capture");
        const cudaError_t le = launch_batched(b, b->capture_stream, accumulate);
        e = cudaStreamEndCapture(b->capture_stream, &b->graph);
        if (le != cudaSuccess)
            return cuda_error(le, "captured launch");
        if (e != cudaSuccess)
            return cuda_error(e, "graph capture end");
        if ((e = cudaGraphInstantiate(&b->graph_exec, b->graph, 0)) != cudaSuccess)
            return cuda_error(e, "graph instantiation");
        b->graph_accumulate = accumulate;
    }
    if ((rc = ctx_begin_timing(ctx)))
        return rc;
    switch (mode) {
    case COUL_BATCH_PERSISTENT:
        e = launch_batched(b, ctx->stream, accumulate);
        break;
    case COUL_BATCH_GRAPH:
        e = cudaGraphLaunch(b->graph_exec, ctx->stream);
        break;
    case COUL_BATCH_SEPARATE: {
        // The baseline: one plain forward launch per molecule, same tile shape.
        coul_tune t = b->tune;
        const VariantEntry* v = nullptr;
        if ((rc = validate_tune(&t, kModeGrid3d, 0, &v)))
            return rc;
        for (const auto& m : b->molecules) {
            FwdParams p{};
            p.atoms = reinterpret_cast<const float4*>(m.d_atoms);
            p.n_atoms = m.n_atoms;
            p.nx = m.grid.nx;
            p.ny = m.grid.ny;
            p.nz = m.grid.nz;
            p.h = m.grid.spacing;
            p.ox = m.grid.origin[0];
            p.oy = m.grid.origin[1];
            p.oz = m.grid.origin[2];
            p.out = m.d_out;
            p.accumulate = accumulate;
            if ((rc = launch_forward(ctx, v, p, kModeGrid3d, &t)))
                return rc;
        }
        break;
    }
    default:
        return set_error(COUL_ERR_INVALID_ARGUMENT, "unknown batch mode");
    }
    if (e != cudaSuccess)
        return cuda_error(e, "batched launch");
    return ctx_end_timing(ctx);
}

}  // extern "C"
