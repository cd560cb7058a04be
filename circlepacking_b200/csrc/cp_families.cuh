// Per-box evaluation of the six lane-packing families in FP64.
//
// One call evaluates one raw box (la, r1_, r2_[, r3]) the way the innermost loop
// of the family's kernel does: tighten r2 by r3.lo and r1 by r2.lo, run the fit
// check, then the guarded criteria.  References (lane_packing/):
//   start          start_configuration.cu:126-162   (handle_case_1/2 :93-111)
//   start_end_2d   start_configuration.cu:200-212   (handle_2d_case  :169-188)
//   start_end_3d   start_configuration.cu:277-295   (handle_3d_case  :227-265)
//   middle         middle_configuration.cu:166-201  (handle_case_1_1/2_1 :86-154)
//   end_2d         end_configuration.cu:109-144     (handle_*_2d     :71-101)
//   end_3d         end_configuration.cu:223-265     (handle_r1_*_3d  :154-210)
//
// Sub-criterion k failing sets bit k of the mask (middle: bits 0/1 are the two
// guarded checks of handle_case_1_1, bits 2/3 those of handle_case_2_1).
// Modes:
//   FULL    every sub-criterion is evaluated; mask and verdict are complete and
//           (optionally) the compared pair (lhs, rhs) of each is traced.
//   DECIDE  stops at the first failing handle (order given by `order`);
//           PROVED / EMPTY are exactly as in FULL, a not-proved box reports the
//           first event met (fit check, trap site or failing handle).
#pragma once
#include "cp_fp64.cuh"

namespace cpb {

struct Verdict {
    uint8_t verdict, mask;
    uint8_t handles;  // guarded criteria (handles) evaluated for this box
};

// The terms of the start family's criteria that do not depend on lambda
// (start_configuration.cu:126-162): the collision angle of disks 1 and 3 on the
// outer border, ca_outer_outer(r1, r3), and the upper semicircle angle of r1.
// They are functions of the radii alone (r1 tightened by r2 and r3), so a box
// whose radii equal its parent's bit for bit has its parent's values.
// flag: 0 = not available, 1 = available, 2 = available and their evaluation
// reached a trap site.
struct LaFree {
    double a13lo, a13hi, so_hi, flag;
};

enum EvalMode { FULL = 0, DECIDE = 1 };

__device__ __forceinline__ void trace_put(double* tr, int k, double lhs, double rhs) {
    if (tr) {
        tr[2 * k] = lhs;
        tr[2 * k + 1] = rhs;
    }
}

// Sub-checks of handle_case_1_1 / handle_case_2_1 (middle_configuration.cu:86-154)
// given the three collision angles; k0 = bit of the first sub-check.  The
// handles are not inlined: one copy each keeps the kernels within the
// instruction caches (measured 6-9% faster on middle and end_3d).
template <int MODE>
__device__ __forceinline__ bool middle_handle(Iv la, Iv r1, Iv r2, Iv r3, bool inner_first, uint8_t& mask, int k0,
                                              bool& trap, double* tr) {
    const double ratio = area_ratio_ub(la);
    const double a1 = disk_area_lb(r1), a2 = disk_area_lb(r2);
    // guard "possibly": c13.lo <= (c12 + c23).hi
    double c12_hi, c23_hi, c13_lo;
    if (inner_first) {
        c12_hi = ca_mixed_hi<false>(la, r1, r2, trap);
        c13_lo = ca_inner_inner_lo(la, r1, r3, trap);
        c23_hi = ca_mixed_hi<true>(la, r2, r3, trap);
    } else {
        c12_hi = ca_mixed_hi<true>(la, r1, r2, trap);
        c13_lo = ca_outer_outer_lo(r1, r3, trap);
        c23_hi = ca_mixed_hi<false>(la, r2, r3, trap);
    }
    bool failed = false;
    if (c13_lo <= __dadd_ru(c12_hi, c23_hi)) {
        double used = used_ub(ratio, c12_hi);
        double lhs = __dmul_rd(0.5, __dadd_rd(a1, a2));
        double rhs = __dmul_ru(kCriticalRatio, used);
        if (MODE == FULL) trace_put(tr, k0, lhs, rhs);
        if (lhs < rhs) {
            mask |= (uint8_t)(1u << k0);
            failed = true;
            if (MODE == DECIDE) return true;
        }
    }
    // guard "possibly not": !(c13.hi <= (c12 + c23).lo)
    double c12_lo, c23_lo, c13_hi;
    if (inner_first) {
        c12_lo = ca_mixed_lo<false>(la, r1, r2, trap);
        c13_hi = ca_inner_inner_hi(la, r1, r3, trap);
        c23_lo = ca_mixed_lo<true>(la, r2, r3, trap);
    } else {
        c12_lo = ca_mixed_lo<true>(la, r1, r2, trap);
        c13_hi = ca_outer_outer_hi(r1, r3, trap);
        c23_lo = ca_mixed_lo<false>(la, r2, r3, trap);
    }
    if (!(c13_hi <= __dadd_rd(c12_lo, c23_lo))) {
        double used = used_ub(ratio, c13_hi);
        double a3 = disk_area_lb(r3);
        double lhs = __dadd_rd(__dmul_rd(0.5, __dadd_rd(a1, a3)), a2);
        double rhs = __dmul_ru(kCriticalRatio, used);
        if (MODE == FULL) trace_put(tr, k0 + 1, lhs, rhs);
        if (lhs < rhs) {
            mask |= (uint8_t)(1u << (k0 + 1));
            failed = true;
        }
    }
    return failed;
}

// handle_inner_outer_2d (INNER) / handle_outer_inner_2d, end_configuration.cu:71-101
template <bool INNER>
__device__ __forceinline__ bool end2d_handle(Iv la, Iv r1, Iv r2, bool& trap, double* lhs_out, double* rhs_out) {
    Iv ca, sa;
    double other_hi, rho_lo;
    if (INNER) {
        ca = ca_inner_outer(la, r1, r2, trap);
        sa = {semi_outer_lo(r2), semi_outer_hi(r2)};
        other_hi = semi_inner_hi(la, r1);
        Iv t = isub(pt(1.0), iscale(2.0, r2));
        rho_lo = __dadd_rd(isq(t).lo, -isq(la).hi);
    } else {
        ca = ca_outer_inner(la, r1, r2, trap);
        sa = {semi_inner_lo(la, r2), semi_inner_hi(la, r2)};
        other_hi = semi_outer_hi(r1);
        rho_lo = __dadd_rd(1.0, -isq(iadd(la, iscale(2.0, r2))).hi);
    }
    Iv a = iadd(ca, sa);
    const double ratio = area_ratio_ub(la);
    const double used = used_ub(ratio, a.hi);
    if (rho_lo < 0.0) rho_lo = 0.0;
    const double alpha = __dadd_rd(a.lo, -other_hi);
    const double reusable = __dmul_rd(__dmul_rd(0.5, alpha), rho_lo);
    const double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
    *lhs_out = __dadd_rd(ar2, __dmul_rd(0.5, ar1));
    *rhs_out = __dmul_ru(kCriticalRatio, __dadd_ru(used, -reusable));
    return !(*lhs_out >= *rhs_out);
}

// handle_r1_inner_3d (INNER) / handle_r1_outer_3d, end_configuration.cu:154-210.
// Returns true when the handle fails; *evaluated = false on the early exit.
template <bool INNER>
__device__ __forceinline__ bool end3d_handle(Iv la, Iv r1, Iv r2, Iv r3, bool& trap, bool* evaluated, double* lhs_out,
                                              double* rhs_out) {
    // early exit: definitely(a12 + a23 >= a13)  <=>  a13.hi <= (a12 + a23).lo
    double a12_lo, a23_lo, a13_hi;
    if (INNER) {
        a12_lo = ca_mixed_lo<false>(la, r1, r2, trap);
        a23_lo = ca_mixed_lo<true>(la, r2, r3, trap);
        a13_hi = ca_inner_inner_hi(la, r1, r3, trap);
    } else {
        a12_lo = ca_mixed_lo<true>(la, r1, r2, trap);
        a23_lo = ca_mixed_lo<false>(la, r2, r3, trap);
        a13_hi = ca_outer_outer_hi(r1, r3, trap);
    }
    // the reference evaluates a23 in full although only a23.lo is consumed: its
    // upper corner can still reach a trap site
    if (INNER)
        ca_mixed_hi<true, true>(la, r2, r3, trap);
    else
        ca_mixed_hi<false, true>(la, r2, r3, trap);
    if (a13_hi <= __dadd_rd(a12_lo, a23_lo)) {
        // early exit (end_configuration.cu:159-162, 188-191); the reference has
        // already evaluated a12.hi and a13.lo at this point
        if (INNER) {
            ca_mixed_hi<false, true>(la, r1, r2, trap);
            ca_inner_inner_lo<true>(la, r1, r3, trap);
        } else {
            ca_mixed_hi<true, true>(la, r1, r2, trap);
            ca_outer_outer_lo<true>(r1, r3, trap);
        }
        *evaluated = false;
        return false;
    }
    *evaluated = true;
    double a12_hi, a13_lo;
    Iv a3;
    double a2_hi, rho_lo;
    if (INNER) {
        a12_hi = ca_mixed_hi<false>(la, r1, r2, trap);
        a13_lo = ca_inner_inner_lo(la, r1, r3, trap);
        a3 = {semi_inner_lo(la, r3), semi_inner_hi(la, r3)};
        a2_hi = semi_outer_hi(r2);
        rho_lo = __dadd_rd(1.0, -isq(iadd(la, iscale(2.0, r3))).hi);
    } else {
        a12_hi = ca_mixed_hi<true>(la, r1, r2, trap);
        a13_lo = ca_outer_outer_lo(r1, r3, trap);
        a3 = {semi_outer_lo(r3), semi_outer_hi(r3)};
        a2_hi = semi_inner_hi(la, r2);
        Iv t = isub(pt(1.0), iscale(2.0, r3));
        rho_lo = __dadd_rd(isq(t).lo, -isq(la).hi);
    }
    Iv a = iadd(Iv{a13_lo, a13_hi}, a3);
    const double reusable_alpha_lo = __dadd_rd(a.lo, -__dadd_ru(a12_hi, a2_hi));
    if (rho_lo < 0.0) rho_lo = 0.0;
    const double reusable = __dmul_rd(__dmul_rd(0.5, reusable_alpha_lo), rho_lo);
    const double ratio = area_ratio_ub(la);
    const double used = used_ub(ratio, a.hi);
    const double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2), ar3 = disk_area_lb(r3);
    *lhs_out = __dadd_rd(__dadd_rd(ar2, ar3), __dmul_rd(0.5, ar1));
    *rhs_out = __dmul_ru(kCriticalRatio, __dadd_ru(used, -reusable));
    return !(*lhs_out >= *rhs_out);
}

// Out-of-line copies of the handles (one each), with every flag and result in
// registers: the bodies above are inlined into these, and each returns what
// its caller needs (flags packed, the compared pair for traces) by value.
struct HandleOut {
    double lhs, rhs;
    uint32_t bits;  // bit 0: failed, bit 1: trap site reached, bit 2: criterion evaluated; bits 8..15: mask
};
template <int MODE>
__device__ __noinline__ HandleOut middle_handle_call(Iv la, Iv r1, Iv r2, Iv r3, bool inner_first, int k0,
                                                     double* tr) {
    uint8_t mask = 0;
    bool trap = false;
    const bool failed = middle_handle<MODE>(la, r1, r2, r3, inner_first, mask, k0, trap, tr);
    return {0.0, 0.0, (failed ? 1u : 0u) | (trap ? 2u : 0u) | ((uint32_t)mask << 8)};
}
template <bool INNER>
__device__ __noinline__ HandleOut end2d_handle_call(Iv la, Iv r1, Iv r2) {
    bool trap = false;
    double lhs = 0.0, rhs = 0.0;
    const bool failed = end2d_handle<INNER>(la, r1, r2, trap, &lhs, &rhs);
    return {lhs, rhs, (failed ? 1u : 0u) | (trap ? 2u : 0u) | 4u};
}
template <bool INNER>
__device__ __noinline__ HandleOut end3d_handle_call(Iv la, Iv r1, Iv r2, Iv r3) {
    bool trap = false, evaluated = false;
    double lhs = 0.0, rhs = 0.0;
    const bool failed = end3d_handle<INNER>(la, r1, r2, r3, trap, &evaluated, &lhs, &rhs);
    return {lhs, rhs, (failed ? 1u : 0u) | (trap ? 2u : 0u) | (evaluated ? 4u : 0u)};
}

// Evaluates one raw box.  lo/hi hold the family's dims axes (la, r1, r2, r3).
// order: for the families with two independent handles (middle, end_2d,
// end_3d) bit 0 set = evaluate the second handle first (DECIDE mode only).
// tr: FULL mode only, 16 doubles (lhs, rhs per sub-criterion) or nullptr.
// la_in / la_out (start family, optional): the lambda-independent terms of this
// box when already known (la_in->flag != 0), and where to report them.
template <int FAM, int MODE>
__device__ __forceinline__ Verdict eval_box(const double* lo, const double* hi, int order, double* tr,
                                            const LaFree* la_in = nullptr, LaFree* la_out = nullptr) {
    constexpr int D = family_dims(FAM);
    Iv la{lo[0], hi[0]}, r1{lo[1], hi[1]}, r2{lo[2], hi[2]}, r3{0.0, 0.0};
    if (D == 4) {
        r3 = {lo[3], hi[3]};
        if (r2.lo < r3.lo) r2.lo = r3.lo;
    }
    if (r1.lo < r2.lo) r1.lo = r2.lo;
    if (iempty(la) || iempty(r1) || iempty(r2) || (D == 4 && iempty(r3))) return {V_EMPTY, 0};

    uint8_t mask = 0;
    uint8_t handles = 0;
    bool trap = false;
    // the start+end kernels have no fit check (start_configuration.cu:190-215, 267-298)
    const bool fit_fires = FAM != F_START_END_2D && FAM != F_START_END_3D &&
                           __dmul_ru(2.0, r1.hi) >= __dadd_rd(1.0, -la.hi);
    if (fit_fires) mask |= M_FIT;
    // middle / end kernels trap on the fit check before any criterion
    if (MODE == DECIDE && fit_fires && FAM != F_START && FAM != F_START_END_2D && FAM != F_START_END_3D)
        return {V_NOFIT, mask};
    double lhs = 0.0, rhs = 0.0;

    if (FAM == F_START) {
        const Iv a12 = ca_outer_inner(la, r1, r2, trap);
        Iv a13;
        double so_hi;
        if (la_in && la_in->flag != 0.0) {
            a13 = {la_in->a13lo, la_in->a13hi};
            so_hi = la_in->so_hi;
            if (la_in->flag == 2.0) trap = true;
            if (la_out) *la_out = *la_in;
        } else {
            bool t13 = false;
            a13 = ca_outer_outer(r1, r3, t13);
            so_hi = semi_outer_hi(r1);
            if (t13) trap = true;
            if (la_out) *la_out = {a13.lo, a13.hi, so_hi, t13 ? 2.0 : 1.0};
        }
        const Iv a23 = ca_inner_outer(la, r2, r3, trap);
        const Iv s = iadd(a12, a23);
        const Ub case1{a13.hi < s.lo, a13.lo < s.hi};  // a12 + a23 > a13
        const double ratio = area_ratio_ub(la);
        const double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
        if (case1.pos) {
            ++handles;
            double used = used_ub(ratio, __dadd_ru(so_hi, a12.hi));
            lhs = __dadd_rd(ar1, __dmul_rd(0.5, ar2));
            rhs = __dmul_ru(kCriticalRatio, used);
            if (MODE == FULL) trace_put(tr, 0, lhs, rhs);
            if (!(lhs >= rhs)) {
                mask |= 1;
                if (MODE == DECIDE) goto done;
            }
        }
        if (!case1.def) {
            ++handles;
            double used = used_ub(ratio, __dadd_ru(so_hi, a13.hi));
            double ar3 = disk_area_lb(r3);
            lhs = __dadd_rd(__dadd_rd(ar1, ar2), __dmul_rd(0.5, ar3));
            rhs = __dmul_ru(kCriticalRatio, used);
            if (MODE == FULL) trace_put(tr, 1, lhs, rhs);
            if (!(lhs >= rhs)) mask |= 2;
        }
    } else if (FAM == F_START_END_2D) {
        handles = 1;
        const double a1_hi = semi_outer_hi(r1);
        const Iv a2{semi_inner_lo(la, r2), semi_inner_hi(la, r2)};
        const Iv a12 = ca_outer_inner(la, r1, r2, trap);
        const double total_hi = __dadd_ru(__dadd_ru(a1_hi, a2.hi), a12.hi);
        double reuse_lo = __dadd_rd(__dadd_rd(a12.lo, a2.lo), -a1_hi);
        if (reuse_lo < 0.0) reuse_lo = 0.0;
        const double ratio = area_ratio_ub(la);
        const double used = used_ub(ratio, total_hi);
        double rho_lo = __dadd_rd(1.0, -isq(iadd(la, iscale(2.0, r2))).hi);
        if (rho_lo < 0.0) rho_lo = 0.0;
        const double reusable = __dmul_rd(__dmul_rd(0.5, reuse_lo), rho_lo);
        const double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
        lhs = __dadd_rd(ar2, ar1);
        rhs = __dmul_ru(kCriticalRatio, __dadd_ru(used, -reusable));
        if (MODE == FULL) trace_put(tr, 0, lhs, rhs);
        if (!(lhs >= rhs)) mask |= 1;
    } else if (FAM == F_START_END_3D) {
        handles = 1;
        const Iv a1{semi_outer_lo(r1), semi_outer_hi(r1)};
        const Iv a2{semi_inner_lo(la, r2), semi_inner_hi(la, r2)};
        const Iv a3{semi_outer_lo(r3), semi_outer_hi(r3)};
        const Iv a12 = ca_outer_inner(la, r1, r2, trap);
        const Iv a13 = ca_outer_outer(r1, r2, trap);  // (r1, r2) as in start_configuration.cu:232
        const Iv a23 = ca_inner_outer(la, r2, r3, trap);
        const Iv b123 = iadd(a12, a23);
        const Iv b13{dmax_lo(a13.lo, b123.lo), dmax_lo(a13.hi, b123.hi)};
        const Iv a123 = iadd(iadd(a1, b13), a3);
        const Iv a122 = iadd(iadd(a1, a12), a2);
        const Iv a{dmax_lo(a123.lo, a122.lo), dmax_lo(a123.hi, a122.hi)};
        double reuse_angle = __dadd_rd(a.lo, -a122.hi);
        if (reuse_angle < 0.0) reuse_angle = 0.0;
        const double outer_rad = __dadd_rd(1.0, -__dmul_ru(2.0, r3.hi));
        const double outer_sq = __dmul_rd(outer_rad, outer_rad);
        const double inner_sq = __dmul_ru(la.hi, la.hi);
        double reused = __dmul_rd(__dmul_rd(0.5, reuse_angle), __dadd_rd(outer_sq, -inner_sq));
        if (reused < 0.0) reused = 0.0;
        const double ratio = area_ratio_ub(la);
        const double used = __dadd_ru(used_ub(ratio, a.hi), -reused);
        const double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2), ar3 = disk_area_lb(r3);
        lhs = __dadd_rd(ar1, __dadd_rd(ar2, ar3));
        rhs = __dmul_ru(kCriticalRatio, used);
        if (MODE == FULL) trace_put(tr, 0, lhs, rhs);
        if (!(lhs >= rhs)) mask |= 1;
    } else if (FAM == F_MIDDLE) {
        const bool second_first = (MODE == DECIDE) && (order & 1);
        for (int h = 0; h < 2; ++h) {
            const bool inner = (h == 0) != second_first;
            ++handles;
            const HandleOut o = middle_handle_call<MODE>(la, r1, r2, r3, inner, inner ? 0 : 2, tr);
            mask |= (uint8_t)(o.bits >> 8);
            if (o.bits & 2u) trap = true;
            const bool failed = (o.bits & 1u) != 0;
            if (MODE == DECIDE && failed) break;
        }
    } else if (FAM == F_END_2D) {
        const bool second_first = (MODE == DECIDE) && (order & 1);
        for (int h = 0; h < 2; ++h) {
            const bool inner = (h == 0) != second_first;
            ++handles;
            const HandleOut o = inner ? end2d_handle_call<true>(la, r1, r2) : end2d_handle_call<false>(la, r1, r2);
            lhs = o.lhs;
            rhs = o.rhs;
            if (o.bits & 2u) trap = true;
            const bool failed = (o.bits & 1u) != 0;
            const int k = inner ? 0 : 1;
            if (MODE == FULL) trace_put(tr, k, lhs, rhs);
            if (failed) {
                mask |= (uint8_t)(1u << k);
                if (MODE == DECIDE) break;
            }
        }
    } else if (FAM == F_END_3D) {
        const bool second_first = (MODE == DECIDE) && (order & 1);
        for (int h = 0; h < 2; ++h) {
            const bool inner = (h == 0) != second_first;
            ++handles;
            bool evaluated = false;
            const HandleOut o =
                inner ? end3d_handle_call<true>(la, r1, r2, r3) : end3d_handle_call<false>(la, r1, r2, r3);
            lhs = o.lhs;
            rhs = o.rhs;
            evaluated = (o.bits & 4u) != 0;
            if (o.bits & 2u) trap = true;
            const bool failed = (o.bits & 1u) != 0;
            const int k = inner ? 0 : 1;
            if (MODE == FULL && evaluated) trace_put(tr, k, lhs, rhs);
            if (failed) {
                mask |= (uint8_t)(1u << k);
                if (MODE == DECIDE) break;
            }
        }
    }
done:
    if (trap) mask |= M_TRAP;
    uint8_t v;
    if (mask & M_TRAP)
        v = V_ERROR;
    else if ((mask & M_FIT) && FAM != F_START && FAM != F_START_END_2D && FAM != F_START_END_3D)
        v = V_NOFIT;
    else if (mask & M_CRIT)
        v = V_CRITICAL;
    else
        v = V_PROVED;
    return {v, mask, handles};
}

}  // namespace cpb
