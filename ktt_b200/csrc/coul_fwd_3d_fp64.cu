// Forward variants: 3D, float4 atoms through TMA-staged shared memory, every pair evaluated in FP64
// (COUL_PREC_FP64_PAIRS: MUFU rsqrt.approx.f64 estimate, one FP64 Newton step, FP64 accumulation).
#include "coul_forward.cuh"

namespace coul {

void register_fwd_3d_fp64(std::vector<VariantEntry>& v)
{
#define COUL_FP64(ZI, XP)                                                                 \
    add_variant<ZI, XP, 1, kSrcShared, 0, kPrecFp64Pairs, 0, kModeGrid3d>(v);             \
    add_variant<ZI, XP, 2, kSrcShared, 0, kPrecFp64Pairs, 0, kModeGrid3d>(v);
    COUL_FP64(4, 1)
    COUL_FP64(4, 2)
    COUL_FP64(4, 4)
    COUL_FP64(8, 1)
    COUL_FP64(8, 2)
    COUL_FP64(8, 4)
    COUL_FP64(16, 1)
    COUL_FP64(16, 2)
#undef COUL_FP64
}

}  // namespace coul
