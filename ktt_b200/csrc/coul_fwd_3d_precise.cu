// Forward variants: 3D, float4 atoms through TMA-staged shared memory, FP32 partials per
// 64-atom sub-tile merged by two-sum (compensated) or into FP64 (FP64 merge).
#include "coul_forward.cuh"

namespace coul {

template <int PREC, int SOFT>
static void add_precise(std::vector<VariantEntry>& v)
{
#define COUL_XP(ZI)                                                                 \
    add_variant<ZI, 1, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);               \
    add_variant<ZI, 1, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);               \
    add_variant<ZI, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);               \
    add_variant<ZI, 2, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);               \
    add_variant<ZI, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);               \
    add_variant<ZI, 4, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    COUL_XP(2)
    COUL_XP(4)
    COUL_XP(8)
    COUL_XP(16)
#undef COUL_XP
}

void register_fwd_3d_precise(std::vector<VariantEntry>& v)
{
    add_precise<kPrecCompensated, 0>(v);
    add_precise<kPrecFp64Merge, 0>(v);
}

}  // namespace coul
