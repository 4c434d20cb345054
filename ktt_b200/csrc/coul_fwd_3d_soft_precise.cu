// Forward variants: 3D, float4 atoms through TMA-staged shared memory, a static share of the
// reciprocal square roots on the FMA pipe, with compensated (two-sum) accumulation.  The FP64-merge
// form of the same shapes is in coul_fwd_3d_soft_fp64m.cu.
#include "coul_soft_precise.cuh"

namespace coul {

void register_fwd_3d_soft_precise(std::vector<VariantEntry>& v)
{
    add_soft_precise_shares<kPrecCompensated>(v);
}

}  // namespace coul
