// Forward variants, atom-split (thread-block cluster) form: for 2D slices and small 3D maps whose
// point tiles alone cannot fill 148 SMs.  A cluster of 2..8 CTAs shares one point tile, each CTA
// streams its own share of the atoms through a TMA ring, and rank 0 reduces the partial blocks
// over distributed shared memory in rank order.  Plain FP32 accumulation, AoS atoms.
#include "coul_forward.cuh"

namespace coul {

template <int ZI, int XP, int SOFT, int MODE>
static void add_split_unrolls(std::vector<VariantEntry>& v)
{
    add_split_variant<ZI, XP, 1, SOFT, MODE>(v);
    add_split_variant<ZI, XP, 2, SOFT, MODE>(v);
    add_split_variant<ZI, XP, 4, SOFT, MODE>(v);
}

void register_fwd_split(std::vector<VariantEntry>& v)
{
    // 2D slice: rows per thread (ZI) x points per thread along x (XP)
    add_split_unrolls<1, 1, 0, kModeSlice2d>(v);
    add_split_unrolls<2, 1, 0, kModeSlice2d>(v);
    add_split_unrolls<4, 1, 0, kModeSlice2d>(v);
    add_split_unrolls<1, 2, 0, kModeSlice2d>(v);
    add_split_unrolls<2, 2, 0, kModeSlice2d>(v);
    add_split_unrolls<2, 1, 2, kModeSlice2d>(v);
    add_split_unrolls<4, 1, 2, kModeSlice2d>(v);
    add_split_unrolls<2, 2, 2, kModeSlice2d>(v);
    // eight points per thread: fewer shared-memory atom loads per rsqrt, and a whole-tile FMA-pipe share
    add_split_unrolls<4, 2, 0, kModeSlice2d>(v);
    add_split_unrolls<4, 2, 2, kModeSlice2d>(v);
    add_split_unrolls<4, 2, 3, kModeSlice2d>(v);
    add_split_unrolls<2, 4, 0, kModeSlice2d>(v);
    add_split_unrolls<2, 4, 2, kModeSlice2d>(v);
    add_split_unrolls<8, 1, 0, kModeSlice2d>(v);
    add_split_unrolls<8, 1, 2, kModeSlice2d>(v);
    add_split_unrolls<2, 2, 3, kModeSlice2d>(v);
    // sixteen points per thread: eight lane pairs, so the FMA-pipe share is taken within each thread
    add_split_unrolls<8, 2, 2, kModeSlice2d>(v);
    add_split_unrolls<8, 2, 3, kModeSlice2d>(v);
    add_split_unrolls<4, 4, 2, kModeSlice2d>(v);
    // 3D map: z points per thread (ZI) x points per thread along x (XP)
    add_split_unrolls<4, 1, 0, kModeGrid3d>(v);
    add_split_unrolls<8, 1, 0, kModeGrid3d>(v);
    add_split_unrolls<8, 2, 0, kModeGrid3d>(v);
    add_split_unrolls<8, 1, 2, kModeGrid3d>(v);
    add_split_unrolls<8, 2, 2, kModeGrid3d>(v);
}

}  // namespace coul
