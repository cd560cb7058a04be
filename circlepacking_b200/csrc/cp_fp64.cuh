// FP64 directed-rounding interval evaluation of the lane-packing criteria.
//
// Semantics follow the reference's device code bit for bit (same CUDA
// intrinsics, same operation order, same CUDA asin), restated for the GPU:
//   * interval ops: algcuda/cuda-utils/cuh/include/algcuda/interval.cuh:38-355
//   * asin padding: interval.cuh:420-438 (5 representable steps outward)
//   * primitives:   lane_packing/collision_angles.cu:29-246
//   * single placement bound: lane_packing/lower_bound_radius_single_placement.cu:26-61
//   * criteria:     lane_packing/{start,middle,end}_configuration.cu
//
// Design differences (results unchanged):
//   * Every collision-angle evaluation at a box corner feeds exactly one bound of
//     its caller (collision_angles.cu:119-231), so `collision<HI>` computes only
//     that bound: 2 asin calls per branch instead of 4.  The emptiness test of
//     the obtuse partial result (collision_angles.cu:108) is decided from the
//     wanted bound alone; this relies on asin_rd(x) <= asin_ru(y) for x <= y,
//     which the 5-step padding guarantees under CUDA's documented 2-ulp asin
//     error bound -- the same bound the reference's padding relies on.
//   * Interval-by-interval multiplication never occurs on this path; squares
//     use the absolute value (interval.hpp:214-231) exactly as the reference.
//   * No printf and no trap: trap sites set a per-box flag (verdict ERROR).
#pragma once
#include <cstdint>

namespace cpb {

// lane_packing/values.hpp:28-32
constexpr double kCriticalRatio = 0.5642;
constexpr double kLbPi = 3.141592653589793;
constexpr double kLambdaMin = 0.5;
constexpr double kLambdaMax = 0.9900000000000001;
// interval.cuh:366 (detail::ub_pi_two)
constexpr double kUbPiTwo = 1.5707963267948968;

// Per-box verdicts and fail-mask bits (shared with the C ABI).
enum : uint8_t { V_PROVED = 0, V_CRITICAL = 1, V_NOFIT = 2, V_EMPTY = 3, V_ERROR = 4 };
enum : uint8_t { M_FIT = 0x40, M_TRAP = 0x80, M_CRIT = 0x3F };
enum Family : int { F_START = 0, F_START_END_2D = 1, F_START_END_3D = 2, F_MIDDLE = 3, F_END_2D = 4, F_END_3D = 5 };

__host__ __device__ constexpr int family_dims(int fam) { return (fam == F_START_END_2D || fam == F_END_2D) ? 3 : 4; }

struct Iv {
    double lo, hi;
};
// Uncertain<bool> (interval.hpp:32-82): def = "definitely", pos = "possibly"
struct Ub {
    bool def, pos;
};

// ------------------------------------------------------------------ asin padding
// IEEE nextafter(y, -2.0) applied five times, for y finite or NaN, |y| < 2.
__device__ __forceinline__ double step_down5(double y) {
    long long b = __double_as_longlong(y);
    if (y > 0.0) {
        // magnitude shrinks; after reaching +0 the steps continue into the negatives
        return b >= 5 ? __longlong_as_double(b - 5) : __longlong_as_double((long long)(0x8000000000000000ull) | (5 - b));
    }
    if (y < 0.0) return __longlong_as_double(b + 5);
    if (y == 0.0) return __longlong_as_double((long long)0x8000000000000005ull);
    return y;  // NaN
}
// IEEE nextafter(y, +2.0) applied five times.
__device__ __forceinline__ double step_up5(double y) {
    long long b = __double_as_longlong(y);
    if (y < 0.0) {
        long long m = b & 0x7fffffffffffffffll;
        return m >= 5 ? __longlong_as_double(b - 5) : __longlong_as_double(5 - m);
    }
    if (y > 0.0) return __longlong_as_double(b + 5);
    if (y == 0.0) return __longlong_as_double(5ll);
    return y;
}
// detail::dasin_rd (interval.cuh:420-428).  Not inlined: CUDA's asin is long and
// is called at ~20 sites per family; one shared copy keeps the level kernels
// within the instruction caches (instruction-fetch stalls dominated otherwise).
static __device__ __noinline__ double asin_rd(double x) {
    double y = step_down5(asin(x));
    if (y < -kUbPiTwo) y = -kUbPiTwo;
    if (x >= 0.0 && y < 0.0) y = 0.0;
    return y;
}
// detail::dasin_ru (interval.cuh:430-438), not inlined (see asin_rd)
static __device__ __noinline__ double asin_ru(double x) {
    double y = step_up5(asin(x));
    if (y > kUbPiTwo) y = kUbPiTwo;
    if (x <= 0.0 && y > 0.0) y = 0.0;
    return y;
}

// ------------------------------------------------------------------ directed division
// a / b rounded down / up, bit-identical to __ddiv_rd / __ddiv_ru.  Method:
// Markstein's FMA division with the rounding direction read off an exact
// remainder.  For |a|, |b| in [2^-500, 2^500]:
//   y0 = rcp.approx(b), e = 1 - b*y0 (one FMA); if |e| >= 2^-18 the intrinsic
//        is used instead.  y = y0 + y0*e then has |1 - b*y| <= e^2 + 2^-52.
//   q0 = a*y;  q = q0 + (a - q0*b)*y   (two FMAs): |q - a/b| stays below half
//        an ulp of q plus ~2^-72 |a/b|, so q is a faithful quotient.
//   r  = a - q*b (one FMA): the exact difference is 0 or a multiple of
//        ~2^-605, so its rounded value has the exact sign.  r = 0: a/b = q;
//        otherwise a/b lies strictly between q and its neighbour on the side
//        of sign(r)*sign(b), which fixes both directed results.
// Operands outside the range (zeros, subnormals, infinities, NaN, extreme
// exponents) use the intrinsics.
__device__ __forceinline__ bool div_in_range(double a, double b) {
    const unsigned ea = ((unsigned)__double2hiint(a) >> 20) & 0x7ffu;
    const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7ffu;
    return (ea - 523u) <= 1000u && (eb - 523u) <= 1000u;
}
// neighbours of a finite, normal, nonzero q (never crossing zero or infinity)
__device__ __forceinline__ double next_up(double q) {
    const long long b = __double_as_longlong(q);
    return __longlong_as_double(q > 0.0 ? b + 1 : b - 1);
}
__device__ __forceinline__ double next_down(double q) {
    const long long b = __double_as_longlong(q);
    return __longlong_as_double(q > 0.0 ? b - 1 : b + 1);
}
// Reciprocal seed: 0 = the FP64 approximation (rcp.approx.ftz.f64), 1 = the
// FP32 reciprocal of b rounded to float (valid for |b| within float range).
template <int SEED>
__device__ __forceinline__ double rcp_seed(double b) {
    double y;
    if (SEED == 0) {
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    } else {
        float yf;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(__double2float_rn(b)));
        y = (double)yf;
    }
    return y;
}
template <bool UP>
static __device__ __noinline__ double div_slow(double a, double b) { return UP ? __ddiv_ru(a, b) : __ddiv_rd(a, b); }
template <bool UP, int SEED = 0>
__device__ __forceinline__ double div_dir(double a, double b) {
    double y = rcp_seed<SEED>(b);
    const double e = __fma_rn(-b, y, 1.0);
    if (!div_in_range(a, b) || !(fabs(e) < 3.814697265625e-06)) return div_slow<UP>(a, b);
    y = __fma_rn(y, e, y);
    const double q0 = __dmul_rn(a, y);
    const double q = __fma_rn(__fma_rn(-q0, b, a), y, q0);
    const double r = __fma_rn(-q, b, a);
    if (r == 0.0) return q;                     // exact quotient
    const bool above = (r > 0.0) != (b < 0.0);  // a/b > q
    if (UP) return above ? next_up(q) : q;
    return above ? q : next_down(q);
}
// Not inlined either: ~66 divisions per box, and one shared copy of each
// direction (with the intrinsic fallback out of line) keeps the level kernels
// small enough for the instruction caches; measured 10-24% faster per family.
static __device__ __noinline__ double div_rd(double a, double b) { return div_dir<false>(a, b); }
static __device__ __noinline__ double div_ru(double a, double b) { return div_dir<true>(a, b); }

// ------------------------------------------------------------------ interval ops
__device__ __forceinline__ Iv pt(double x) { return {x, x}; }
__device__ __forceinline__ Iv iadd(Iv a, Iv b) { return {__dadd_rd(a.lo, b.lo), __dadd_ru(a.hi, b.hi)}; }
__device__ __forceinline__ Iv isub(Iv a, Iv b) { return {__dadd_rd(a.lo, -b.hi), __dadd_ru(a.hi, -b.lo)}; }
// scalar * interval for the non-negative powers of two used here: both bounds
// rounded down as in interval.cuh:185-190 (exact for these scalars)
__device__ __forceinline__ Iv iscale(double n, Iv a) { return {__dmul_rd(a.lo, n), __dmul_rd(a.hi, n)}; }
// interval.hpp:214-231 + interval.cuh:352-355
__device__ __forceinline__ Iv isq(Iv x) {
    double l = 0.0, u = 0.0;
    if (x.hi > 0)
        u = x.hi;
    else
        l = -x.hi;
    if (x.lo < 0)
        u = u < -x.lo ? -x.lo : u;
    else
        l = x.lo;
    return {__dmul_rd(l, l), __dmul_ru(u, u)};
}
// interval.cuh:277-310, one bound at a time
__device__ __forceinline__ double idiv_lo(Iv a, Iv o) {
    if (o.lo > 0) return a.lo >= 0 ? div_rd(a.lo, o.hi) : div_rd(a.lo, o.lo);
    if (o.hi < 0) return (a.lo >= 0 || !(a.hi <= 0)) ? div_rd(a.hi, o.hi) : div_rd(a.hi, o.lo);
    return -__longlong_as_double(0x7ff0000000000000ll);
}
__device__ __forceinline__ double idiv_hi(Iv a, Iv o) {
    if (o.lo > 0) return (a.lo >= 0 || !(a.hi <= 0)) ? div_ru(a.hi, o.lo) : div_ru(a.hi, o.hi);
    if (o.hi < 0) return a.lo >= 0 ? div_ru(a.lo, o.lo) : div_ru(a.lo, o.hi);
    return __longlong_as_double(0x7ff0000000000000ll);
}
__device__ __forceinline__ Iv idiv(Iv a, Iv o) { return {idiv_lo(a, o), idiv_hi(a, o)}; }
__device__ __forceinline__ bool iempty(Iv a) { return a.lo > a.hi; }
__device__ __forceinline__ double dmax_lo(double a, double b) { return a < b ? b : a; }  // "a < b ? b : a"

// ------------------------------------------------------------------ collision angle
// x / o takes the positive branches of the interval division (o.lo > 0,
// x.lo >= 0), both intervals are proper, and the lower-end quotient's operands
// lie in the certified division's range (so an FMA remainder has an exact sign).
__device__ __forceinline__ bool posq(Iv x, Iv o) {
    return o.lo > 0.0 && x.lo >= 0.0 && x.lo <= x.hi && o.lo <= o.hi && div_in_range(x.lo, o.hi);
}
// RD(a / b) > 1 for a >= 0, b > 0 in range: a / b >= 1 + 2^-52, i.e. the exact
// a - b * (1 + 2^-52) is not negative (one FMA; its rounding keeps the sign).
__device__ __forceinline__ bool rd_quot_gt1(double a, double b) {
    return __fma_rn(-b, 1.0000000000000002, a) >= 0.0;
}

// What a caller needs from compute_collision_angle: one bound, or only whether
// a trap site is reached (for corners the reference evaluates but whose value no
// criterion consumes; every trap condition is decided before any asin).
enum Want : int { W_LO = 0, W_HI = 1, W_TRAP = 2 };

// compute_collision_angle (collision_angles.cu:37-117) for one Want.
__device__ __forceinline__ double collision_body(Iv L, Iv S, Iv ab, const int W, bool& trap) {
    const bool HI = (W == W_HI);
    if (L.lo < S.lo) L.lo = S.lo;
    if (L.hi < S.hi) S.hi = L.hi;
    const Iv l2 = isq(L), s2 = isq(S), a2 = isq(ab);
    const Iv sum = iadd(s2, a2);
    const Ub obt{sum.hi < l2.lo, sum.lo < l2.hi};
    Iv add = idiv(isub(l2, s2), ab);
    if (add.lo < 0.0) add.lo = 0.0;

    // the partial result after the obtuse branch: none ({0,-1}) or [ob_lo, ob_hi]
    bool ob_set = false;
    double ob_val = HI ? -1.0 : 0.0;  // wanted bound of the partial result
    // for LO: what is needed to decide emptiness of the partial result lazily
    Iv lq{0, 0}, sq{0, 0};
    bool lq_hi_lazy = false;
    double ob_lx_hi = 0.0, ob_sx_lo = 0.0;

    // Quotients whose only use is an emptiness or a domain test are not
    // computed when an exact comparison decides that test (positive, proper
    // operands in the certified division's range: `posq`).  For such x / o:
    //   RD(x.lo / o.hi) > 1  <=>  x.lo >= o.hi * (1 + 2^-52)  (rd_quot_gt1)
    //   RU(x.hi / o.lo) > 1  <=>  x.hi > o.lo
    //   RD(x.lo / o.hi) >= 0 > -1,  and the quotient interval is proper.
    // Every value and every trap decision is the one of the full evaluation.
    if (obt.pos) {
        Iv lx = iscale(0.5, iadd(add, ab));
        Iv sx = iscale(0.5, isub(add, ab));
        if (sx.lo < 0.0) sx.lo = 0.0;
        if (S.hi < sx.hi) sx.hi = S.hi;
        if (L.hi < lx.hi) lx.hi = L.hi;
        if (iempty(sx) || iempty(lx)) {
            if (obt.def) trap = true;
        } else if (posq(lx, L) && posq(sx, S)) {
            // lq = lx / L, sq = sx / S: proper, non-negative; after clamping the
            // upper ends to 1, empty iff the lower end exceeds 1; no domain trap
            if (W == W_TRAP) {
                if (rd_quot_gt1(lx.lo, L.hi) || rd_quot_gt1(sx.lo, S.hi)) {
                    if (obt.def) trap = true;
                } else {
                    ob_set = true;
                }
            } else if (HI) {
                double lqh = div_ru(lx.hi, L.lo);
                if (1.0 < lqh) lqh = 1.0;
                const double sql = div_rd(sx.lo, S.hi);
                if (rd_quot_gt1(lx.lo, L.hi) || sql > 1.0) {
                    if (obt.def) trap = true;
                } else {
                    ob_set = true;
                    ob_val = __dadd_ru(asin_ru(lqh), -asin_rd(sql));
                }
            } else {
                const double lql = div_rd(lx.lo, L.hi);
                double sqh = div_ru(sx.hi, S.lo);
                if (1.0 < sqh) sqh = 1.0;
                if (lql > 1.0 || rd_quot_gt1(sx.lo, S.hi)) {
                    if (obt.def) trap = true;
                } else {
                    ob_set = true;
                    lq.lo = lql;
                    sq.hi = sqh;
                    lq_hi_lazy = true;  // lq.hi and sq.lo: computed only if the join needs them
                    ob_lx_hi = lx.hi;
                    ob_sx_lo = sx.lo;
                    ob_val = __dadd_rd(asin_rd(lql), -asin_ru(sqh));
                    if (ob_val < 0.0) ob_val = 0.0;
                }
            }
        } else {
            lq = idiv(lx, L);
            if (1.0 < lq.hi) lq.hi = 1.0;
            sq = idiv(sx, S);
            if (1.0 < sq.hi) sq.hi = 1.0;
            if (iempty(lq) || iempty(sq)) {
                if (obt.def) trap = true;
            } else {
                if (lq.lo < -1.0 || lq.hi > 1.0 || sq.lo < -1.0 || sq.hi > 1.0) trap = true;
                ob_set = true;
                if (W == W_TRAP) {
                } else if (HI) {
                    ob_val = __dadd_ru(asin_ru(lq.hi), -asin_rd(sq.lo));
                } else {
                    ob_val = __dadd_rd(asin_rd(lq.lo), -asin_ru(sq.hi));
                    if (ob_val < 0.0) ob_val = 0.0;
                }
            }
        }
    }

    if (!obt.def) {
        Iv lx = iscale(0.5, iadd(ab, add));
        Iv sx = iscale(0.5, isub(ab, add));
        if (sx.lo < 0.0) sx.lo = 0.0;
        if (iempty(sx)) {
            if (!obt.pos) trap = true;
        } else {
            const bool fast = posq(lx, L) && posq(sx, S);
            if (W == W_TRAP) {
                if (fast) {
                    if (lx.hi > L.lo || sx.hi > S.lo) trap = true;
                } else {
                    Iv alq = idiv(lx, L), asq = idiv(sx, S);
                    if (alq.lo < -1.0 || alq.hi > 1.0 || asq.lo < -1.0 || asq.hi > 1.0) trap = true;
                }
                return 0.0;
            }
            double r;
            if (HI) {
                double lqh = idiv_hi(lx, L), sqh = idiv_hi(sx, S);
                if (lqh > 1.0 || sqh > 1.0) trap = true;
                if (!(lx.lo >= 0.0 && L.lo > 0.0) && idiv_lo(lx, L) < -1.0) trap = true;
                if (!(sx.lo >= 0.0 && S.lo > 0.0) && idiv_lo(sx, S) < -1.0) trap = true;
                r = __dadd_ru(asin_ru(lqh), asin_ru(sqh));
            } else {
                double alql, asql;
                if (fast) {
                    alql = div_rd(lx.lo, L.hi);
                    asql = div_rd(sx.lo, S.hi);
                    if (lx.hi > L.lo || sx.hi > S.lo) trap = true;
                } else {
                    Iv alq = idiv(lx, L), asq = idiv(sx, S);
                    if (alq.lo < -1.0 || alq.hi > 1.0 || asq.lo < -1.0 || asq.hi > 1.0) trap = true;
                    alql = alq.lo;
                    asql = asq.lo;
                }
                double b = asin_rd(asql);
                if (b < 0.0) b = 0.0;
                r = __dadd_rd(asin_rd(alql), b);
            }
            // result.empty() ? result = r : result.do_join(r)   (collision_angles.cu:108-112)
            bool ob_nonempty;
            if (!ob_set) {
                ob_nonempty = false;
            } else if (HI) {
                ob_nonempty = !(ob_val < 0.0);
            } else {
                if (lq_hi_lazy) {
                    lq.hi = div_ru(ob_lx_hi, L.lo);
                    if (1.0 < lq.hi) lq.hi = 1.0;
                    sq.lo = div_rd(ob_sx_lo, S.hi);
                }
                // empty  <=>  ru(asin_ru(lq.hi) - asin_rd(sq.lo)) < 0, which cannot hold when lq.hi >= sq.lo
                ob_nonempty = (lq.hi >= sq.lo) || !(__dadd_ru(asin_ru(lq.hi), -asin_rd(sq.lo)) < 0.0);
            }
            if (!ob_nonempty)
                ob_val = r;
            else if (HI ? (r > ob_val) : (r < ob_val))
                ob_val = r;
        }
    }
    return ob_val;
}

// The trap flag is a register of the out-of-line function and comes back with
// the value: a flag passed by reference into an out-of-line function would
// live in local memory.
struct DTrap {
    double v;
    bool trap;
};
// One copy for all three Wants (a runtime argument): the three template
// copies of this long routine were the largest part of the level kernels'
// instruction footprint.
static __device__ __noinline__ DTrap collision_call(Iv L, Iv S, Iv ab, int W) {
    bool trap = false;
    const double v = collision_body(L, S, ab, W, trap);
    return {v, trap};
}
template <int W>
__device__ __forceinline__ double collision(Iv L, Iv S, Iv ab, bool& trap) {
    const DTrap r = collision_call(L, S, ab, W);
    trap = trap || r.trap;
    return r.v;
}

// collision_angles.cu:119-142.  TRAP_ONLY: evaluate only the trap sites.
template <bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_inner_inner_hi(Iv la, Iv ra, Iv rb, bool& trap) {
    Iv lc{__dadd_rd(ra.hi, la.lo), __dadd_ru(ra.hi, la.lo)};
    Iv sc{__dadd_rd(rb.hi, la.lo), __dadd_ru(rb.hi, la.lo)};
    Iv ab{__dadd_rd(ra.hi, rb.hi), __dadd_ru(ra.hi, rb.hi)};
    return collision<TRAP_ONLY ? W_TRAP : W_HI>(lc, sc, ab, trap);
}
template <bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_inner_inner_lo(Iv la, Iv ra, Iv rb, bool& trap) {
    Iv lc{__dadd_rd(ra.lo, la.hi), __dadd_ru(ra.lo, la.hi)};
    Iv sc{__dadd_rd(rb.lo, la.hi), __dadd_ru(rb.lo, la.hi)};
    Iv ab{__dadd_rd(ra.lo, rb.lo), __dadd_ru(ra.lo, rb.lo)};
    if (ab.lo <= 0.0) return 0.0;
    return collision<TRAP_ONLY ? W_TRAP : W_LO>(lc, sc, ab, trap);
}
// collision_angles.cu:207-231
template <bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_outer_outer_hi(Iv ra, Iv rb, bool& trap) {
    Iv lc{__dadd_rd(1.0, -rb.hi), __dadd_ru(1.0, -rb.hi)};
    Iv sc{__dadd_rd(1.0, -ra.hi), __dadd_ru(1.0, -ra.hi)};
    Iv ab{__dadd_rd(ra.hi, rb.hi), __dadd_ru(ra.hi, rb.hi)};
    return collision<TRAP_ONLY ? W_TRAP : W_HI>(lc, sc, ab, trap);
}
template <bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_outer_outer_lo(Iv ra, Iv rb, bool& trap) {
    Iv lc{__dadd_rd(1.0, -rb.lo), __dadd_ru(1.0, -rb.lo)};
    Iv sc{__dadd_rd(1.0, -ra.lo), __dadd_ru(1.0, -ra.lo)};
    Iv ab{__dadd_rd(ra.lo, rb.lo), __dadd_ru(ra.lo, rb.lo)};
    if (ab.lo <= 0.0) return 0.0;
    return collision<TRAP_ONLY ? W_TRAP : W_LO>(lc, sc, ab, trap);
}
// collision_angles.cu:144-158 and 175-189 for point radii a, b: the disk
// touching the outer border has centre distance 1-a (OUTER_FIRST) or 1-b.
template <int W, bool OUTER_FIRST>
__device__ __forceinline__ double ca_mixed_corner(Iv la, double a, double b, bool& trap) {
    Iv ca, cb;
    if (OUTER_FIRST) {
        ca = {__dadd_rd(1.0, -a), __dadd_ru(1.0, -a)};
        cb = {__dadd_rd(la.lo, b), __dadd_ru(la.hi, b)};
    } else {
        ca = {__dadd_rd(la.lo, a), __dadd_ru(la.hi, a)};
        cb = {__dadd_rd(1.0, -b), __dadd_ru(1.0, -b)};
    }
    Iv ab{__dadd_rd(a, b), __dadd_ru(a, b)};
    const bool def_ca_longer = cb.hi <= ca.lo;
    const bool pos_ca_longer = cb.lo <= ca.hi;
    // one call site for the first (or only) ordering, so the lanes of a warp
    // that take different orderings evaluate it together
    const bool swap = !def_ca_longer && !pos_ca_longer;  // cb is definitely the longer side
    const double r1 = collision<W>(swap ? cb : ca, swap ? ca : cb, ab, trap);
    if (def_ca_longer || swap) return r1;
    const double r2 = collision<W>(cb, ca, ab, trap);
    return (W == W_HI) ? (r2 > r1 ? r2 : r1) : (r2 < r1 ? r2 : r1);
}
// collision_angles.cu:160-173 (OUTER_FIRST) and 191-205: lower bound is 0 when
// the disks possibly fit side by side across the lane.
template <bool OUTER_FIRST, bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_mixed_lo(Iv la, Iv ra, Iv rb, bool& trap) {
    double lhs_lo = __dmul_rd(__dadd_rd(ra.lo, rb.lo), 2.0);
    double rhs_hi = __dadd_ru(1.0, -la.lo);
    if (lhs_lo <= rhs_hi) return 0.0;
    return ca_mixed_corner<TRAP_ONLY ? W_TRAP : W_LO, OUTER_FIRST>(la, ra.lo, rb.lo, trap);
}
template <bool OUTER_FIRST, bool TRAP_ONLY = false>
__device__ __forceinline__ double ca_mixed_hi(Iv la, Iv ra, Iv rb, bool& trap) {
    return ca_mixed_corner<TRAP_ONLY ? W_TRAP : W_HI, OUTER_FIRST>(la, ra.hi, rb.hi, trap);
}
__device__ __forceinline__ Iv ca_inner_inner(Iv la, Iv ra, Iv rb, bool& t) {
    double hi = ca_inner_inner_hi(la, ra, rb, t);
    return {ca_inner_inner_lo(la, ra, rb, t), hi};
}
__device__ __forceinline__ Iv ca_outer_outer(Iv ra, Iv rb, bool& t) {
    double hi = ca_outer_outer_hi(ra, rb, t);
    return {ca_outer_outer_lo(ra, rb, t), hi};
}
__device__ __forceinline__ Iv ca_outer_inner(Iv la, Iv ra, Iv rb, bool& t) {
    return {ca_mixed_lo<true>(la, ra, rb, t), ca_mixed_hi<true>(la, ra, rb, t)};
}
__device__ __forceinline__ Iv ca_inner_outer(Iv la, Iv ra, Iv rb, bool& t) {
    return {ca_mixed_lo<false>(la, ra, rb, t), ca_mixed_hi<false>(la, ra, rb, t)};
}
// collision_angles.cu:233-246, one bound at a time
__device__ __forceinline__ double semi_outer_lo(Iv r) { return asin_rd(div_rd(r.lo, __dadd_ru(1.0, -r.lo))); }
__device__ __forceinline__ double semi_outer_hi(Iv r) { return asin_ru(div_ru(r.hi, __dadd_rd(1.0, -r.hi))); }
__device__ __forceinline__ double semi_inner_lo(Iv la, Iv r) { return asin_rd(div_rd(r.lo, __dadd_ru(la.hi, r.lo))); }
__device__ __forceinline__ double semi_inner_hi(Iv la, Iv r) { return asin_ru(div_ru(r.hi, __dadd_rd(la.lo, r.hi))); }

// lower_bound_radius_single_placement.cu:26-61: bisection for the smallest
// radius r with r^2/asin(r/(1-r)) >= (critical_ratio/pi) (1 - lambda^2).
__device__ inline double single_placement(double lb_lambda) {
    const double f = div_ru(kCriticalRatio, kLbPi);
    const double rhs = __dmul_ru(f, __dadd_ru(1.0, -__dmul_rd(lb_lambda, lb_lambda)));
    double ub = 0.25, lb = 5.0e-324;
    for (int it = 0; it < 2100; ++it) {
        double mid = __dmul_rn(0.5, __dadd_rn(lb, ub));
        if (mid <= lb || mid >= ub) return ub;
        double r_sq = __dmul_rd(mid, mid);
        double q = div_ru(mid, __dadd_rd(1.0, -mid));
        double lhs = div_rd(r_sq, asin_ru(q));
        if (lhs >= rhs)
            ub = mid;
        else
            lb = mid;
    }
    return ub;
}

// ------------------------------------------------------------------ shared terms
__device__ __forceinline__ double area_ratio_ub(Iv la) { return __dadd_ru(1.0, -__dmul_rd(la.lo, la.lo)); }
__device__ __forceinline__ double disk_area_lb(Iv r) { return __dmul_rd(kLbPi, __dmul_rd(r.lo, r.lo)); }
__device__ __forceinline__ double used_ub(double ratio, double angle_hi) {
    return __dmul_ru(ratio, __dmul_ru(0.5, angle_hi));
}

}  // namespace cpb
