// Forward variants, atom-split queue form: for 2D slices and small 3D maps, a persistent grid claims
// (point tile, atom chunk) items from a device queue and the CTA that finishes a tile's last chunk
// adds its partial blocks from device memory in chunk order.  Plain FP32 accumulation, AoS atoms.
#include "coul_forward.cuh"

namespace coul {

template <int ZI, int XP, int SOFT, int MODE>
static void add_queue_unrolls(std::vector<VariantEntry>& v)
{
    add_queue_split_variant<ZI, XP, 1, SOFT, MODE>(v);
    add_queue_split_variant<ZI, XP, 2, SOFT, MODE>(v);
}

void register_fwd_queue_split(std::vector<VariantEntry>& v)
{
    // 2D slice: rows per thread (ZI) x points per thread along x (XP)
    add_queue_unrolls<2, 2, 0, kModeSlice2d>(v);
    add_queue_unrolls<2, 2, 2, kModeSlice2d>(v);
    add_queue_unrolls<4, 1, 2, kModeSlice2d>(v);
    add_queue_unrolls<4, 2, 0, kModeSlice2d>(v);
    add_queue_unrolls<4, 2, 2, kModeSlice2d>(v);
    add_queue_unrolls<4, 2, 3, kModeSlice2d>(v);
    add_queue_unrolls<2, 4, 2, kModeSlice2d>(v);
    add_queue_unrolls<8, 2, 2, kModeSlice2d>(v);
    add_queue_unrolls<4, 4, 2, kModeSlice2d>(v);
    // 3D map
    add_queue_unrolls<8, 1, 2, kModeGrid3d>(v);
    add_queue_unrolls<8, 2, 2, kModeGrid3d>(v);
    add_queue_unrolls<4, 2, 2, kModeGrid3d>(v);
}

}  // namespace coul
