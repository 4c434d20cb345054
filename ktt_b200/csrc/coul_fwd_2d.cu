// Forward variants: 2D slice in KTT's 2D argument convention (atom .z = dz^2), float4 atoms
// through TMA-staged shared memory, plain FP32, all-MUFU.  Points per thread along x
// (KTT OUTER_UNROLL_FACTOR) {1, 2, 4, 8} x rows per thread along y {1, 2, 4, 8}.
#include "coul_forward.cuh"

namespace coul {

void register_fwd_2d(std::vector<VariantEntry>& v)
{
#define COUL_XP(YI)                                                        \
    add_unrolls<YI, 1, kSrcShared, 0, kPrecFp32, 0, kModeSlice2d>(v);      \
    add_unrolls<YI, 2, kSrcShared, 0, kPrecFp32, 0, kModeSlice2d>(v);      \
    add_unrolls<YI, 4, kSrcShared, 0, kPrecFp32, 0, kModeSlice2d>(v);      \
    add_unrolls<YI, 8, kSrcShared, 0, kPrecFp32, 0, kModeSlice2d>(v);
    COUL_XP(1)
    COUL_XP(2)
    COUL_XP(4)
    COUL_XP(8)
#undef COUL_XP
}

}  // namespace coul
