// FP32 enclosure pre-pass (filled in below).
#pragma once
#include "cp_fp64.cuh"

namespace cpb {
enum PrefilterResult { PF_UNDECIDED = 0, PF_PROVED = 1, PF_EMPTY = 2 };
template <int FAM>
__device__ __forceinline__ int prefilter_box(const double* lo, const double* hi) {
    return PF_UNDECIDED;
}
}  // namespace cpb
