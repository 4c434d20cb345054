// Forward variants: 3D, float4 atoms through TMA-staged shared memory, a static share of the
// reciprocal square roots on the FMA pipe, FP32 sub-tile partials merged into FP64 sums kept in shared
// memory instead of registers (the FP64-merge arithmetic with fewer registers per thread).
#include "coul_soft_precise.cuh"

namespace coul {

void register_fwd_3d_soft_fp64s(std::vector<VariantEntry>& v)
{
    add_soft_precise_shares<kPrecFp64MergeShared>(v);
    add_soft_precise<kPrecFp64MergeShared, 0>(v);
}

}  // namespace coul
