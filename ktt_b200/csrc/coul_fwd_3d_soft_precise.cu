// Forward variants: 3D, float4 atoms through TMA-staged shared memory, a static share of the
// reciprocal square roots on the FMA pipe, with compensated (two-sum) or FP64-merge accumulation.
#include "coul_forward.cuh"

namespace coul {

template <int PREC, int SOFT>
static void add_soft_precise(std::vector<VariantEntry>& v)
{
    add_variant<8, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 1, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<4, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
}

template <int PREC>
static void add_shares(std::vector<VariantEntry>& v)
{
    add_soft_precise<PREC, 1>(v);
    add_soft_precise<PREC, 2>(v);
    add_soft_precise<PREC, 3>(v);
}

void register_fwd_3d_soft_precise(std::vector<VariantEntry>& v)
{
    add_shares<kPrecCompensated>(v);
    add_shares<kPrecFp64Merge>(v);
}

}  // namespace coul
