// Forward variants: 3D, float4 atoms through TMA-staged shared memory, with a static share of the
// reciprocal square roots (SOFT of every 8 lane pairs, or from kSoftAlternate on an alternation of two
// neighbouring eighths over consecutive atoms) evaluated by Newton iterations on the FMA pipe so the
// MUFU unit and the FMA pipe are both busy.  Plain FP32 accumulation (the compensated
// and FP64-merge forms are in coul_fwd_3d_soft_precise.cu).
#include "coul_forward.cuh"

namespace coul {

template <int PREC, int SOFT>
static void add_soft(std::vector<VariantEntry>& v)
{
    add_variant<4, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<4, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 1, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 1, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<4, 1, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 2, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 1, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 1, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<32, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
}

template <int PREC>
static void add_soft_shares(std::vector<VariantEntry>& v)
{
    add_soft<PREC, 1>(v);
    add_soft<PREC, 2>(v);
    add_soft<PREC, 3>(v);
    add_soft<PREC, 4>(v);
    add_soft<PREC, 5>(v);
    // alternating shares between the eighths: 3/16 and 5/16 of the lane pairs
    add_soft<PREC, kSoftAlternate + 1>(v);
    add_soft<PREC, kSoftAlternate + 2>(v);
}

void register_fwd_3d_soft(std::vector<VariantEntry>& v)
{
    add_soft_shares<kPrecFp32>(v);
}

}  // namespace coul
