// Forward variants: 3D, float4 atoms through TMA-staged shared memory, a static share of the
// reciprocal square roots on the FMA pipe, FP32 sub-tile partials merged into FP64.
#include "coul_soft_precise.cuh"

namespace coul {

void register_fwd_3d_soft_fp64m(std::vector<VariantEntry>& v)
{
    add_soft_precise_shares<kPrecFp64Merge>(v);
}

}  // namespace coul
