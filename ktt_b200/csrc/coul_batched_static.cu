// coul_batched_static.cu -- the batched persistent map with its scratch in a static device array.
//
// coul_batch_create keeps the molecule table and the work-queue counter in device memory it
// allocates with cudaMalloc.  Some callers cannot let a library allocate device memory: a host
// application that hands all free device memory to its own pool allocator at start-up (so a late
// cudaMalloc fails or fragments that pool), or a latency-critical loop that cannot afford the
// implicit device synchronisation of cudaFree, or a plug-in whose host forbids allocation outside
// its own allocator.  coul_batch_run_static serves them: the same persistent kernel, with its
// scratch -- the queue counter and the molecule table -- in g_batch_scratch below, a file-scope
// static __device__ array of fixed size that every GPU loading the library holds until exit.  The
// caller passes the atoms and output maps (and an optional status word) as usual; the call makes no
// cudaMalloc or cudaFree and no allocating library call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "coul_batched.cuh"
#include "coul_internal.h"

namespace coul {

// Maximum batch size of the static path and the layout of its scratch: the 64-bit queue counter at
// offset 0, the molecule table from offset 256.
constexpr int kStaticMaxMolecules = 1024;
constexpr size_t kStaticTableOffset = 256;
constexpr size_t kStaticScratchBytes = kStaticTableOffset + sizeof(MolDesc) * kStaticMaxMolecules;

static __device__ __align__(256) unsigned char g_batch_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxDevices = 64;

struct StaticVariant {
    int zi, xp, unroll, prec, soft;
    const void* kernel;
};

template <int ZI, int XP, int UNR, int PREC, int SOFT>
StaticVariant static_variant()
{
    return StaticVariant{ZI, XP, UNR, PREC, SOFT, reinterpret_cast<const void*>(&batched_kernel<ZI, XP, UNR, PREC, SOFT>)};
}

constexpr int kStaticVariants = 3;

const StaticVariant* static_variants()
{
    static const StaticVariant v[kStaticVariants] = {
        static_variant<8, 2, 2, kPrecFp32, 2>(),
        static_variant<8, 2, 1, kPrecFp32, 0>(),
        static_variant<16, 1, 1, kPrecFp32, 2>(),
    };
    return v;
}

// SM count per device, found at the first call on that device (occupancy is looked up per block
// shape on each call).  The scratch array's device address is not cached: a module-scope
// __device__ array has one instance per CUDA context that loads the module, so the address belongs
// to the context current at the call (the device's primary context, or a caller-owned one).
int g_sm_count[kMaxDevices];

std::mutex g_mutex;
MolDesc g_host_table[kStaticMaxMolecules];  // host staging, reused by every call (under g_mutex)
int g_order[kStaticMaxMolecules];

int fail(int status, const char* message)
{
    return set_error(status, message);
}

}  // namespace
}  // namespace coul

using namespace coul;

extern "C" COUL_API int coul_batch_run_static(void* stream, const coul_molecule* molecules, int n_molecules,
                                              const coul_tune* tune, int accumulate, int* d_status)
{
    if (n_molecules < 0 || n_molecules > kStaticMaxMolecules)
        return fail(COUL_ERR_INVALID_ARGUMENT,
                    "coul_batch_run_static: n_molecules must be in 0..1024 (the size of its static molecule table)");
    if (tune == nullptr || (n_molecules > 0 && molecules == nullptr))
        return fail(COUL_ERR_INVALID_ARGUMENT, "coul_batch_run_static: NULL tune or molecules");
    const int threads = tune->block_x * tune->block_y;
    if (tune->block_x < 1 || tune->block_y < 1 || threads > kMaxThreads)
        return fail(COUL_ERR_DEVICE_LIMITS, "coul_batch_run_static: block shape outside 1..256 threads");
    const int unroll = tune->unroll <= 1 ? 1 : tune->unroll;
    const StaticVariant* variant = nullptr;
    for (int i = 0; i < kStaticVariants; ++i) {
        const StaticVariant& v = static_variants()[i];
        if (v.zi == tune->z_iterations && v.xp == tune->x_points && v.unroll == unroll && v.prec == tune->precision &&
            v.soft == tune->rsqrt_soft)
            variant = &v;
    }
    if (variant == nullptr || tune->atom_source != COUL_ATOMS_SHARED_TMA)
        return fail(COUL_ERR_UNSUPPORTED,
                    "coul_batch_run_static: tile shape not compiled for the static path (z_iterations/x_points/"
                    "unroll/precision/rsqrt_soft = 8/2/2/0/2, 8/2/1/0/0 or 16/1/1/0/2)");
    for (int i = 0; i < n_molecules; ++i) {
        const coul_molecule& m = molecules[i];
        if (validate_grid(&m.grid) != COUL_OK)
            return COUL_ERR_INVALID_ARGUMENT;
        if (m.n_atoms < 0 || m.d_out == nullptr || (m.n_atoms > 0 && (m.d_atoms == nullptr || !aligned16(m.d_atoms))))
            return fail(COUL_ERR_INVALID_ARGUMENT, "coul_batch_run_static: bad atoms or output pointer");
        if (m.grid.nx > (1 << 24) || m.grid.ny > (1 << 24) || m.grid.nz > (1 << 24))
            return fail(COUL_ERR_INVALID_ARGUMENT, "coul_batch_run_static: grid too large");
    }

    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return cuda_error(e, "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices)
        return fail(COUL_ERR_NO_DEVICE, "coul_batch_run_static: device index beyond 63");

    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_sm_count[device] == 0) {
        int sm = 0;
        if ((e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
            return cuda_error(e, "cudaDeviceGetAttribute");
        g_sm_count[device] = sm;
    }
    // The device address of the static scratch array in the context current on this thread (in
    // host code the symbol itself is only a host-side stand-in).  A lookup, no allocation; the first
    // lookup in a context loads this library's device code into it.
    void* scratch_ptr = nullptr;
    if ((e = cudaGetSymbolAddress(&scratch_ptr, g_batch_scratch)) != cudaSuccess)
        return cuda_error(e, "cudaGetSymbolAddress of the static batch scratch");
    unsigned char* scratch = static_cast<unsigned char*>(scratch_ptr);

    // Molecule table in decreasing order of pair count (same work list as coul_batch_create).
    for (int i = 0; i < n_molecules; ++i)
        g_order[i] = i;
    auto pairs = [&](int i) {
        const coul_molecule& m = molecules[i];
        return static_cast<double>(m.grid.nx) * m.grid.ny * m.grid.nz * static_cast<double>(m.n_atoms);
    };
    std::stable_sort(g_order, g_order + n_molecules, [&](int a, int c) { return pairs(a) > pairs(c); });
    int64_t next = 0;
    coul_tune t = *tune;
    t.unroll = unroll;
    for (int k = 0; k < n_molecules; ++k) {
        MolDesc d{};
        d.tile_begin = next;
        next += fill_mol_desc(d, molecules[g_order[k]], t);
        g_host_table[k] = d;
    }
    if (n_molecules == 0 || next == 0)
        return COUL_OK;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(scratch);
    MolDesc* table = reinterpret_cast<MolDesc*>(scratch + kStaticTableOffset);
    // The copy reads the pageable host table before it returns, so the table may be refilled by the
    // next call; the counter must start at zero.
    if ((e = cudaMemcpyAsync(table, g_host_table, sizeof(MolDesc) * n_molecules, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
        return cuda_error(e, "molecule table upload");
    if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s)) != cudaSuccess)
        return cuda_error(e, "queue counter reset");

    const size_t smem = kStages * kTileAtoms * 16 + kStages * 8;
    int blocks_per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, variant->kernel, threads, smem)) !=
        cudaSuccess)
        return cuda_error(e, "occupancy query");
    if (blocks_per_sm < 1)
        return fail(COUL_ERR_DEVICE_LIMITS, "coul_batch_run_static: kernel does not fit on an SM");
    BatchParams p{table, n_molecules, next, counter, accumulate ? 1 : 0, d_status};
    void* args[] = {&p};
    e = cudaLaunchKernel(variant->kernel, dim3(static_cast<unsigned>(blocks_per_sm * g_sm_count[device])),
                         dim3(static_cast<unsigned>(tune->block_x), static_cast<unsigned>(tune->block_y), 1), args, smem,
                         s);
    if (e != cudaSuccess)
        return cuda_error(e, "static batched launch");
    return COUL_OK;
}
