// Forward variants, atom-split balanced form: for 2D slices and small 3D maps, a resident grid
// whose CTAs take equal contiguous ranges of the (point tile, atom) space, the atom groups of a
// CTA sharing each tile's points; tiles split between CTAs are finished from device memory by the
// CTA that adds their last piece.  Plain FP32 accumulation, AoS atoms.
#include "coul_forward.cuh"

namespace coul {

template <int ZI, int XP, int SOFT, int MODE>
static void add_balanced_unrolls(std::vector<VariantEntry>& v)
{
    add_balanced_split_variant<ZI, XP, 1, SOFT, MODE>(v);
    add_balanced_split_variant<ZI, XP, 2, SOFT, MODE>(v);
}

void register_fwd_balanced_split(std::vector<VariantEntry>& v)
{
    // 2D slice: rows per thread (ZI) x points per thread along x (XP)
    add_balanced_unrolls<4, 2, 0, kModeSlice2d>(v);
    add_balanced_unrolls<4, 2, 2, kModeSlice2d>(v);
    add_balanced_unrolls<4, 2, 3, kModeSlice2d>(v);
    add_balanced_unrolls<2, 2, 2, kModeSlice2d>(v);
    add_balanced_unrolls<8, 2, 2, kModeSlice2d>(v);
    add_balanced_unrolls<4, 4, 2, kModeSlice2d>(v);
    add_balanced_unrolls<4, 4, 3, kModeSlice2d>(v);
    add_balanced_unrolls<4, 4, 12, kModeSlice2d>(v);
    add_balanced_unrolls<8, 2, 3, kModeSlice2d>(v);
    add_balanced_unrolls<8, 2, 12, kModeSlice2d>(v);
    add_balanced_unrolls<2, 4, 2, kModeSlice2d>(v);
    add_balanced_unrolls<8, 1, 2, kModeSlice2d>(v);
    // 3D map
    add_balanced_unrolls<8, 1, 2, kModeGrid3d>(v);
    add_balanced_unrolls<8, 2, 2, kModeGrid3d>(v);
    add_balanced_unrolls<4, 2, 2, kModeGrid3d>(v);
}

}  // namespace coul
