// Forward variants: 3D, atoms as four float arrays (KTT USE_SOA = 1) through TMA-staged shared
// memory, plain FP32, all-MUFU.
#include "coul_forward.cuh"

namespace coul {

void register_fwd_3d_soa(std::vector<VariantEntry>& v)
{
#define COUL_XP(ZI)                                                        \
    add_unrolls<ZI, 1, kSrcShared, 1, kPrecFp32, 0, kModeGrid3d>(v);       \
    add_unrolls<ZI, 2, kSrcShared, 1, kPrecFp32, 0, kModeGrid3d>(v);       \
    add_unrolls<ZI, 4, kSrcShared, 1, kPrecFp32, 0, kModeGrid3d>(v);
    COUL_XP(1)
    COUL_XP(2)
    COUL_XP(4)
    COUL_XP(8)
    COUL_XP(16)
    COUL_XP(32)
#undef COUL_XP
}

}  // namespace coul
