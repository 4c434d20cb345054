// coul_batched.cuh -- the persistent batched kernel (see coul_batched.cu for the design).
#pragma once

#include "coul_forward.cuh"

namespace coul {

struct MolDesc {
    const float4* atoms;
    int64_t n_atoms;
    float* out;
    int64_t tile_begin;  // first work item of this molecule
    int nx, ny, nz;
    int tiles_x, tiles_y;
    int vec_ok;
    float h, ox, oy, oz;
};

struct BatchParams {
    const MolDesc* mols;
    int n_mol;
    int64_t total_items;
    unsigned long long* counter;
    int accumulate;
    int* status;
};

// One CTA per resident slot; each claims (molecule, tile) work items from b.counter until the
// queue is empty and runs them through tile_pass, the TMA atom ring carrying over between items.
template <int ZI, int XP, int UNR, int PREC, int SOFT>
__global__ void __launch_bounds__(kMaxThreads) batched_kernel(const BatchParams b)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kTileAtoms * 16);
    __shared__ long long s_item;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    ring_init(full, tid);
    uint32_t gstage = 0;

    for (;;) {
        if (tid == 0)
            s_item = static_cast<long long>(atomicAdd(b.counter, 1ull));
        __syncthreads();
        const long long item = s_item;
        __syncthreads();
        if (item >= b.total_items)
            return;

        // the molecule: last one whose first item is <= item
        int lo = 0, hi = b.n_mol - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (b.mols[mid].tile_begin <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const MolDesc m = b.mols[lo];
        const long long local = item - m.tile_begin;
        const int tile_x = static_cast<int>(local % m.tiles_x);
        const long long rest = local / m.tiles_x;
        const int tile_y = static_cast<int>(rest % m.tiles_y);
        const int tile_z = static_cast<int>(rest / m.tiles_y);

        FwdParams p{};
        p.atoms = m.atoms;
        p.n_atoms = m.n_atoms;
        p.nx = m.nx;
        p.ny = m.ny;
        p.nz = m.nz;
        p.h = m.h;
        p.ox = m.ox;
        p.oy = m.oy;
        p.oz = m.oz;
        p.out = m.out;
        p.accumulate = b.accumulate;
        p.status = b.status;
        const int x0 = (tile_x * blockDim.x + threadIdx.x) * XP;
        const int yrow = tile_y * blockDim.y + threadIdx.y;
        const int z0 = tile_z * ZI;
        if (!tile_pass<ZI, XP, UNR, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(p, x0, yrow, z0, m.vec_ok, smem_raw, full,
                                                                              gstage))
            return;
    }
}

}  // namespace coul
