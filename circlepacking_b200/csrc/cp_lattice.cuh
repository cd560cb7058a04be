// Lattice box generation: the nested subdivision the reference's family
// kernels enumerate (e.g. middle_configuration.cu:157-168): lambda is the i-th
// of n subintervals of the outer lambda interval and each radius the i-th
// subinterval of its range, which depends on the enclosing coordinates.
#pragma once
#include "cp_fp64.cuh"

namespace cpb {

// get_subinterval (subintervals.hpp:31-42).  nvcc contracts the reference's
// `lb + diff * i` into one fused multiply-add; the explicit __fma_rn keeps the
// same bits here (checked against the reference's own device code).
__device__ __forceinline__ Iv subinterval(Iv iv, int i, int n) {
    double diff = __ddiv_rn(__dadd_rn(iv.hi, -iv.lo), (double)n);
    double l = __fma_rn(diff, (double)i, iv.lo);
    double u = (i + 1 == n) ? iv.hi : __fma_rn(diff, (double)(i + 1), iv.lo);
    return {l, u};
}

// compute_r1_range (start_configuration.cu:58-66; identical in the middle and
// end files): [ (1-la)/4 rounded down, min((1-la)/2, single placement bound) ].
// Scalar products use the reference's rounding (both bounds rounded down).
__device__ __forceinline__ Iv range_r1(Iv la, double single) {
    const double om_lo = __dadd_rd(1.0, -la.hi), om_hi = __dadd_ru(1.0, -la.lo);
    const double ub_lane = __dmul_rd(om_hi, 0.5);
    const double lb_lane = __dmul_rd(om_lo, 0.25);
    return {lb_lane, ub_lane < single ? ub_lane : single};
}
// (0.25*(1-la)).lb, shared by several ranges
__device__ __forceinline__ double quarter_lane_lo(Iv la) { return __dmul_rd(__dadd_rd(1.0, -la.hi), 0.25); }
// (0.5*(1 - la - 2 r)).lb  (start_configuration.cu:74-77, 84-87)
__device__ __forceinline__ double half_gap_lo(Iv la, Iv r) {
    return __dmul_rd(__dadd_rd(__dadd_rd(1.0, -la.hi), -__dmul_rd(r.hi, 2.0)), 0.5);
}
// end_configuration.cu:65-69, 148-152
__device__ __forceinline__ double end_gap_lo(Iv la, Iv r) {
    double lb = __dmul_rd(0.5, __dadd_rd(1.0, -__dadd_ru(la.hi, __dmul_ru(2.0, r.hi))));
    return lb < 0.0 ? 0.0 : lb;
}
__device__ __forceinline__ Iv range_r2(int fam, Iv la, Iv r1) {
    if (fam == F_START_END_2D) return {half_gap_lo(la, r1), r1.hi};
    if (fam == F_END_2D || fam == F_END_3D) return {end_gap_lo(la, r1), r1.hi};
    return {quarter_lane_lo(la), r1.hi};
}
__device__ __forceinline__ Iv range_r3(int fam, Iv la, Iv r2) {
    if (fam == F_START_END_3D) return {half_gap_lo(la, r2), r2.hi};
    if (fam == F_END_3D) return {end_gap_lo(la, r2), r2.hi};
    return {quarter_lane_lo(la), r2.hi};
}

struct LatticeSpec {
    int fam;
    int n[4];
    double outer_lo, outer_hi;
};

// Raw box at lattice coordinates ix; `single` = single placement bound of la.lo.
// Returns false for the boxes the family kernel never visits: end_3d skips the
// whole r3 loop when the r3 range is empty (end_configuration.cu:225-227); the
// subdivision of such a range can still produce a non-empty-looking box.
__device__ __forceinline__ bool lattice_box(const LatticeSpec& s, const int* ix, double single, double* lo, double* hi) {
    const Iv la = subinterval(Iv{s.outer_lo, s.outer_hi}, ix[0], s.n[0]);
    const Iv r1 = subinterval(range_r1(la, single), ix[1], s.n[1]);
    const Iv r2 = subinterval(range_r2(s.fam, la, r1), ix[2], s.n[2]);
    lo[0] = la.lo, hi[0] = la.hi;
    lo[1] = r1.lo, hi[1] = r1.hi;
    lo[2] = r2.lo, hi[2] = r2.hi;
    if (family_dims(s.fam) == 4) {
        const Iv r3r = range_r3(s.fam, la, r2);
        const Iv r3 = subinterval(r3r, ix[3], s.n[3]);
        lo[3] = r3.lo, hi[3] = r3.hi;
        if (s.fam == F_END_3D && iempty(r3r)) return false;
    }
    return true;
}

}  // namespace cpb
