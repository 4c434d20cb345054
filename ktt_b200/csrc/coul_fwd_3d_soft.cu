// Forward variants: 3D, float4 atoms through TMA-staged shared memory, with a static share of the
// reciprocal square roots (SOFT of every 8) evaluated by Newton iterations on the FMA pipe so the
// MUFU unit and the FMA pipe are both busy.  Plain FP32 and FP64-merge accumulation.
#include "coul_forward.cuh"

namespace coul {

template <int PREC, int SOFT>
static void add_soft(std::vector<VariantEntry>& v)
{
    add_variant<8, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
}

void register_fwd_3d_soft(std::vector<VariantEntry>& v)
{
    add_soft<kPrecFp32, 2>(v);
    add_soft<kPrecFp32, 3>(v);
    add_soft<kPrecFp32, 4>(v);
    add_soft<kPrecFp64Merge, 2>(v);
    add_soft<kPrecFp64Merge, 3>(v);
    add_soft<kPrecFp64Merge, 4>(v);
}

}  // namespace coul
