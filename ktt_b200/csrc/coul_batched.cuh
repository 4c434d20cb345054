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
    int tiles_x, tiles_y;  // x-y tiles (tiles_y is 1: the x-y tiles are linear)
    int pitch;             // row length of the x-y numbering: nx rounded up to a multiple of x_points
    int vec_ok;
    float h, ox, oy, oz;
};

// Tile geometry of one molecule.  The x-y tiles are linear: the plane is numbered row by row with
// rows of `pitch` points (nx rounded up to a multiple of x_points, so a thread's x_points points never
// cross a row), and thread i of x-y tile j takes the x_points points from (j * threads + i) * x_points.
// Only the plane's last tile, and for an nx that x_points does not divide the padding column(s), hold
// points outside the grid (evaluated, not stored).  Each point keeps its position x mod x_points in
// its thread, so it is computed exactly as in a one-CTA-per-tile launch.  Returns the molecule's work
// items.
inline int64_t fill_mol_desc(MolDesc& d, const coul_molecule& m, const coul_tune& t)
{
    const int threads = t.block_x * t.block_y;
    const int xp = t.x_points;
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
    d.pitch = (m.grid.nx + xp - 1) / xp * xp;
    const int64_t span = static_cast<int64_t>(threads) * xp;
    d.tiles_x = static_cast<int>((static_cast<int64_t>(d.pitch) * m.grid.ny + span - 1) / span);
    d.tiles_y = 1;
    const int tiles_z = (m.grid.nz + t.z_iterations - 1) / t.z_iterations;
    d.vec_ok = (xp > 1 && m.grid.nx % xp == 0 &&
                (reinterpret_cast<uintptr_t>(m.d_out) % (sizeof(float) * (xp >= 4 ? 4 : xp))) == 0)
                   ? 1
                   : 0;
    return static_cast<int64_t>(d.tiles_x) * tiles_z;
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
        const int tile_z = static_cast<int>(local / m.tiles_x);

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
        // linear x-y tile: points past the plane's last row land at y >= ny, padding columns at
        // x >= nx (evaluated, not stored)
        const int64_t p0 = (static_cast<int64_t>(tile_x) * (blockDim.x * blockDim.y) + tid) * XP;
        const int x0 = static_cast<int>(p0 % m.pitch);
        const int yrow = static_cast<int>(p0 / m.pitch);
        const int z0 = tile_z * ZI;
        // tiles that overhang the molecule's grid in z evaluate only their points inside it
        if (!tile_pass<ZI, XP, UNR, kSrcShared, 0, PREC, SOFT, kModeGrid3d, true>(p, x0, yrow, z0, m.vec_ok,
                                                                                    smem_raw, full, gstage))
            return;
    }
}

}  // namespace coul
