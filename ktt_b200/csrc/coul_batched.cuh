// coul_batched.cuh -- the persistent batched kernel (see coul_batched.cu for the design).
#pragma once

#include "coul_forward.cuh"
#include "coul_internal.h"

namespace coul {

struct MolDesc {
    const float4* atoms;
    int64_t n_atoms;
    float* out;
    int64_t tile_begin;  // first work item of this molecule
    int nx, ny, nz;
    int tiles_x, tiles_y;
    int tx;              // threads of a CTA along x for this molecule's tiles (the rest along y);
                         // 0: linear tiles (one x-y point per thread, consecutive in the x-y plane)
    int vec_ok;
    float h, ox, oy, oz;
};

// Tile geometry of one molecule.  With one x point per thread (x_points 1) the tiles are linear:
// thread i of x-y tile j takes the point j * threads + i of the grid's x-y plane in row-major order,
// so only the plane's last tile is padded.  Otherwise the CTA threads are arranged as
// tx x (threads / tx), tx the power of two dividing the thread count whose tile pads the grid's x-y
// plane least (ties: the block's own x size).  The arrangement only moves points between threads;
// every point is computed the same way.  Returns the molecule's work items.
inline int64_t fill_mol_desc(MolDesc& d, const coul_molecule& m, const coul_tune& t)
{
    const int threads = t.block_x * t.block_y;
    int best_tx = t.block_x;
    int64_t best_area = -1;
    for (int tx = 1; tx <= threads && t.x_points > 1; tx *= 2) {
        if (threads % tx)
            continue;
        const int64_t sx = static_cast<int64_t>(tx) * t.x_points;
        const int64_t sy = threads / tx;
        const int64_t area = (m.grid.nx + sx - 1) / sx * sx * ((m.grid.ny + sy - 1) / sy * sy);
        if (best_area < 0 || area < best_area || (area == best_area && tx == t.block_x)) {
            best_area = area;
            best_tx = tx;
        }
    }
    d.atoms = reinterpret_cast<const float4*>(m.d_atoms);
    d.n_atoms = m.n_atoms;
    d.out = m.d_out;
    d.nx = m.grid.nx;
    d.ny = m.grid.ny;
    d.nz = m.grid.nz;
    d.h = m.grid.spacing;
    d.ox = m.grid.origin[0];
    d.oy = m.grid.origin[1];
    d.oz = m.grid.origin[2];
    if (t.x_points == 1) {
        d.tx = 0;
        d.tiles_x = static_cast<int>((static_cast<int64_t>(m.grid.nx) * m.grid.ny + threads - 1) / threads);
        d.tiles_y = 1;
    } else {
        d.tx = best_tx;
        const int64_t span_x = static_cast<int64_t>(best_tx) * t.x_points;
        const int ty = threads / best_tx;
        d.tiles_x = static_cast<int>((m.grid.nx + span_x - 1) / span_x);
        d.tiles_y = (m.grid.ny + ty - 1) / ty;
    }
    const int tiles_z = (m.grid.nz + t.z_iterations - 1) / t.z_iterations;
    const int xp = t.x_points;
    d.vec_ok = (xp > 1 && m.grid.nx % xp == 0 &&
                (reinterpret_cast<uintptr_t>(m.d_out) % (sizeof(float) * (xp >= 4 ? 4 : xp))) == 0)
                   ? 1
                   : 0;
    return static_cast<int64_t>(d.tiles_x) * d.tiles_y * tiles_z;
}

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
__global__ void __launch_bounds__(kMaxThreads, fwd_min_blocks(PREC, XP * ZI)) batched_kernel(const BatchParams b)
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
        int x0, yrow;
        if (XP == 1 && m.tx == 0) {
            // linear tile: plane points beyond the last row land at y >= ny (evaluated, not stored)
            const int64_t q = static_cast<int64_t>(tile_x) * (blockDim.x * blockDim.y) + tid;
            x0 = static_cast<int>(q % m.nx);
            yrow = static_cast<int>(q / m.nx);
        } else {
            const int ty = static_cast<int>(blockDim.x * blockDim.y) / m.tx;
            x0 = (tile_x * m.tx + tid % m.tx) * XP;
            yrow = tile_y * ty + tid / m.tx;
        }
        const int z0 = tile_z * ZI;
        // tiles that overhang the molecule's grid in z evaluate only their points inside it
        if (!tile_pass<ZI, XP, UNR, kSrcShared, 0, PREC, SOFT, kModeGrid3d, true>(p, x0, yrow, z0, m.vec_ok,
                                                                                    smem_raw, full, gstage))
            return;
    }
}

}  // namespace coul
