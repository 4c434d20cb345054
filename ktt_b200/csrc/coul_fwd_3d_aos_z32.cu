// Forward variants: 3D, float4 atoms through TMA-staged shared memory, plain FP32, all-MUFU,
// Z_ITERATIONS 32 (the largest register blocks, kept in their own translation unit).
#include "coul_forward.cuh"

namespace coul {

void register_fwd_3d_aos_z32(std::vector<VariantEntry>& v)
{
    add_unrolls<32, 1, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);
    add_unrolls<32, 2, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);
    add_unrolls<32, 4, kSrcShared, 0, kPrecFp32, 0, kModeGrid3d>(v);
}

}  // namespace coul
