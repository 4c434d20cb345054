// Forward variants: 3D, atoms as float4 through TMA-staged shared memory, plain FP32, all-MUFU.
// Z_ITERATIONS 1..16 x points-per-thread {1, 2, 4} x atom-loop unroll {1, 2, 4, 8}.
#include "coul_forward.cuh"

namespace coul {

void register_fwd_3d_aos(std::vector<VariantEntry>& v)
{
#define COUL_XP(ZI)                                                        \
    add_unrolls<ZI, 1, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);       \
    add_unrolls<ZI, 2, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);       \
    add_unrolls<ZI, 4, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);
    COUL_XP(1)
    COUL_XP(2)
    COUL_XP(4)
    COUL_XP(8)
    COUL_XP(16)
#undef COUL_XP
}

}  // namespace coul
