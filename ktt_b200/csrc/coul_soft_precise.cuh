// coul_soft_precise.cuh -- the tile shapes and FMA-pipe shares compiled for the precise
// accumulation forms (compensated, FP64 merge) with part of the rsqrts on the FMA pipe; one
// translation unit per form instantiates them.
#pragma once

#include "coul_forward.cuh"

namespace coul {

template <int PREC, int SOFT>
void add_soft_precise(std::vector<VariantEntry>& v)
{
    add_variant<8, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 2, 2, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<8, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 1, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<16, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<4, 2, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
    add_variant<4, 4, 1, kSrcShared, 0, PREC, SOFT, kModeGrid3d>(v);
}

template <int PREC>
void add_soft_precise_shares(std::vector<VariantEntry>& v)
{
    add_soft_precise<PREC, 1>(v);
    add_soft_precise<PREC, 2>(v);
    add_soft_precise<PREC, 3>(v);
    add_soft_precise<PREC, kSoftAlternate + 1>(v);
    add_soft_precise<PREC, kSoftAlternate + 2>(v);
}

}  // namespace coul
