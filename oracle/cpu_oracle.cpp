// TEST INFRASTRUCTURE ONLY -- the CPU oracle.
//
// A CPU restatement of the lane-packing subinterval search of
// phillip-keldenich/circlepacking: the FP64 directed-rounding interval type,
// the geometric primitives, the six families' criteria and dependent ranges,
// the lattice box generation and the lambda refinement loop.  Every function
// cites the reference file:line it restates (paths relative to the
// reference's code/ directory).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
// arm load this library, and only as the checker.  The product library
// (circlepacking_b200/_lib/libcp_b200.so) never links or calls it.
//
// Directed rounding is derived from round-to-nearest results with error-free
// transformations (Knuth's TwoSum for +/-, the FMA product residual for *,
// the FMA division remainder for /), so no rounding-mode switches are needed
// and the library is thread safe.  Operands near the under/overflow limits
// take a <cfenv> slow path.  asin comes from the host libm and is padded by
// the same 5 ulps as the reference, so asin-derived bounds enclose the true
// value but are not bit-identical to the GPU's.
#include <atomic>
#include <cfenv>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <queue>
#include <mutex>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- op counting
struct OpCount {
    uint64_t add, mul, div, asin;
};
static thread_local OpCount* t_count = nullptr;
#define ORC_COUNT(f)           \
    do {                       \
        if (t_count) ++t_count->f; \
    } while (0)

// trap sites reached while evaluating the current box (reference: algcuda::trap)
static thread_local bool t_trap = false;
// Reference-kernel path (op counting only): stop at the first failing
// sub-check of a handle and at the first failing handle of a box, and at the fit
// check where the kernel traps (middle_configuration.cu:173-199,
// end_configuration.cu:115-144, 236-265, start_configuration.cu:141-162).
static thread_local bool t_decide = false;

// ---------------------------------------------------------------- rounding
static inline uint64_t bits_of(double x) {
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
}
static inline double from_bits(uint64_t b) {
    double x;
    std::memcpy(&x, &b, 8);
    return x;
}
// IEEE 754 nextUp / nextDown.
static inline double next_up(double x) {
    if (x != x || x == INFINITY) return x;
    if (x == 0.0) return 0x1p-1074;
    uint64_t b = bits_of(x);
    return from_bits(x > 0.0 ? b + 1 : b - 1);
}
static inline double next_down(double x) { return -next_up(-x); }

enum { OP_ADD = 0, OP_MUL = 1, OP_DIV = 2 };

// Slow path: evaluate one operation under an explicit rounding mode.
__attribute__((noinline)) static double slow_op(int op, bool up, double a, double b) {
    int old = std::fegetround();
    std::fesetround(up ? FE_UPWARD : FE_DOWNWARD);
    volatile double va = a, vb = b;
    volatile double r;
    if (op == OP_ADD)
        r = va + vb;
    else if (op == OP_MUL)
        r = va * vb;
    else
        r = va / vb;
    double out = r;
    std::fesetround(old);
    return out;
}

static const double kSafeLo = 0x1p-900, kSafeHi = 0x1p900;
static inline bool safe_mag(double x) {
    double m = std::fabs(x);
    return m >= kSafeLo && m <= kSafeHi;
}

static inline double add_dir(double a, double b, bool up) {
    double s = a + b;
    if (!std::isfinite(s)) {
        if (std::isfinite(a) && std::isfinite(b)) return slow_op(OP_ADD, up, a, b);
        return s;
    }
    if (s == 0.0) {
        // An exactly-zero sum: IEEE 754 sign rules for the directed modes.
        if (a == 0.0 && b == 0.0) {
            bool na = std::signbit(a), nb = std::signbit(b);
            return up ? ((na && nb) ? -0.0 : 0.0) : ((na || nb) ? -0.0 : 0.0);
        }
        return up ? 0.0 : -0.0;
    }
    double bb = s - a;
    double err = (a - (s - bb)) + (b - bb);
    if (up) return err > 0.0 ? next_up(s) : s;
    return err < 0.0 ? next_down(s) : s;
}

static inline double mul_dir(double a, double b, bool up) {
    double p = a * b;
    if (a == 0.0 || b == 0.0 || !std::isfinite(a) || !std::isfinite(b)) return p;
    if (!safe_mag(p)) return slow_op(OP_MUL, up, a, b);
    double e = std::fma(a, b, -p);
    if (up) return e > 0.0 ? next_up(p) : p;
    return e < 0.0 ? next_down(p) : p;
}

static inline double div_dir(double a, double b, bool up) {
    double q = a / b;
    if (a == 0.0 || b == 0.0 || !std::isfinite(a) || !std::isfinite(b)) return q;
    if (!safe_mag(q) || !safe_mag(a) || !safe_mag(b)) return slow_op(OP_DIV, up, a, b);
    double r = std::fma(-q, b, a);  // exact remainder a - q*b
    bool q_above = (b > 0.0) ? (r < 0.0) : (r > 0.0);
    bool q_below = (b > 0.0) ? (r > 0.0) : (r < 0.0);
    if (up) return q_below ? next_up(q) : q;
    return q_above ? next_down(q) : q;
}

// __dadd_rd/ru, __dmul_rd/ru, __ddiv_rd/ru
static inline double add_rd(double a, double b) { ORC_COUNT(add); return add_dir(a, b, false); }
static inline double add_ru(double a, double b) { ORC_COUNT(add); return add_dir(a, b, true); }
static inline double mul_rd(double a, double b) { ORC_COUNT(mul); return mul_dir(a, b, false); }
static inline double mul_ru(double a, double b) { ORC_COUNT(mul); return mul_dir(a, b, true); }
static inline double div_rd(double a, double b) { ORC_COUNT(div); return div_dir(a, b, false); }
static inline double div_ru(double a, double b) { ORC_COUNT(div); return div_dir(a, b, true); }

// algcuda/cuda-utils/cuh/include/algcuda/interval.cuh:366 (detail::ub_pi_two)
static const double kUbPiTwo = 1.5707963267948968;

// detail::dasin_rd  (interval.cuh:420-428): libm asin, 5 ulps down, clamp.
static inline double asin_rd(double x) {
    ORC_COUNT(asin);
    double y = std::asin(x);
    for (int i = 0; i < 5; ++i) y = std::nextafter(y, -2.0);
    if (y < -kUbPiTwo) y = -kUbPiTwo;
    if (x >= 0.0 && y < 0.0) y = 0.0;
    return y;
}
// detail::dasin_ru  (interval.cuh:430-438)
static inline double asin_ru(double x) {
    ORC_COUNT(asin);
    double y = std::asin(x);
    for (int i = 0; i < 5; ++i) y = std::nextafter(y, 2.0);
    if (y > kUbPiTwo) y = kUbPiTwo;
    if (x <= 0.0 && y > 0.0) y = 0.0;
    return y;
}

// ---------------------------------------------------------------- intervals
// algcuda/cuda-utils/cpp/include/algcuda/interval.hpp:84-242 (Interval<double>)
struct Iv {
    double lb, ub;
};
// interval.hpp:32-82 (Uncertain<bool>): lb = "definitely", ub = "possibly"
struct Ub {
    bool lb, ub;
};
static inline bool definitely(Ub b) { return b.lb; }
static inline bool possibly(Ub b) { return b.ub; }
static inline Ub unot(Ub b) { return {!b.ub, !b.lb}; }

static inline Iv pt(double x) { return {x, x}; }
// interval.cuh:45-51, 58-62: + rounds outward
static inline Iv iadd(Iv a, Iv b) { return {add_rd(a.lb, b.lb), add_ru(a.ub, b.ub)}; }
// interval.cuh:79-85: - rounds outward
static inline Iv isub(Iv a, Iv b) { return {add_rd(a.lb, -b.ub), add_ru(a.ub, -b.lb)}; }
// interval.cuh:185-197: interval * scalar; for n >= 0 BOTH bounds are rounded
// down (exact for the powers of two the prover uses).
static inline Iv iscale(double n, Iv a) {
    if (n >= 0) return {mul_rd(a.lb, n), mul_rd(a.ub, n)};
    double l = mul_rd(a.ub, n), u = mul_ru(a.lb, n);
    return {l, u};
}
// interval.hpp:214-231 (abs)
static inline Iv iabs(Iv a) {
    double l = 0.0, u = 0.0;
    if (a.ub > 0)
        u = a.ub;
    else
        l = -a.ub;
    if (a.lb < 0)
        u = u < -a.lb ? -a.lb : u;
    else
        l = a.lb;
    return {l, u};
}
// interval.cuh:352-355 (square)
static inline Iv isquare(Iv x) {
    Iv a = iabs(x);
    return {mul_rd(a.lb, a.lb), mul_ru(a.ub, a.ub)};
}
// interval.cuh:277-310 (operator/=)
static inline Iv idiv(Iv a, Iv o) {
    double l, u;
    if (o.lb > 0) {
        if (a.lb >= 0) {
            l = div_rd(a.lb, o.ub);
            u = div_ru(a.ub, o.lb);
        } else if (a.ub <= 0) {
            l = div_rd(a.lb, o.lb);
            u = div_ru(a.ub, o.ub);
        } else {
            l = div_rd(a.lb, o.lb);
            u = div_ru(a.ub, o.lb);
        }
    } else if (o.ub < 0) {
        if (a.lb >= 0) {
            l = div_rd(a.ub, o.ub);
            u = div_ru(a.lb, o.lb);
        } else if (a.ub <= 0) {
            l = div_rd(a.ub, o.lb);
            u = div_ru(a.lb, o.ub);
        } else {
            l = div_rd(a.ub, o.ub);
            u = div_ru(a.lb, o.ub);
        }
    } else {
        u = INFINITY;
        l = -u;
    }
    return {l, u};
}
// interval.hpp:134-170 comparisons
static inline Ub ilt(Iv a, Iv b) { return {a.ub < b.lb, a.lb < b.ub}; }
static inline Ub ile(Iv a, Iv b) { return {a.ub <= b.lb, a.lb <= b.ub}; }
static inline Ub igt(Iv a, Iv b) { return ilt(b, a); }
static inline Ub ige(Iv a, Iv b) { return ile(b, a); }
// interval.hpp:197-211
static inline void tighten_lb(Iv& a, double x) {
    if (a.lb < x) a.lb = x;
}
static inline void tighten_ub(Iv& a, double x) {
    if (x < a.ub) a.ub = x;
}
static inline bool iempty(Iv a) { return a.lb > a.ub; }
// interval.hpp:186-195 (do_join)
static inline void ijoin(Iv& a, Iv o) {
    if (o.lb < a.lb) a.lb = o.lb;
    if (o.ub > a.ub) a.ub = o.ub;
}
// interval.cuh:617-624 (asin(Interval)); out-of-range traps in the reference
static inline Iv iasin(Iv x) {
    if (x.lb < -1.0 || x.ub > 1.0) t_trap = true;
    return {asin_rd(x.lb), asin_ru(x.ub)};
}

// ---------------------------------------------------------------- constants
// lane_packing/values.hpp:28-32
static const double kCriticalRatio = 0.5642;
static const double kLbPi = 3.141592653589793;
static const double kLambdaMin = 0.5;
static const double kLambdaMax = 0.9900000000000001;

// ---------------------------------------------------------------- primitives
// collision_angles.cu:29-31
static inline Ub is_obtuse(Iv hyp, Iv s1, Iv s2) {
    return igt(isquare(hyp), iadd(isquare(s1), isquare(s2)));
}

// collision_angles.cu:37-117 (compute_collision_angle)
static Iv collision_angle(Iv longer, Iv shorter, Iv ab) {
    tighten_lb(longer, shorter.lb);
    tighten_ub(shorter, longer.ub);
    Iv result{0.0, -1.0};
    Ub obt = is_obtuse(longer, shorter, ab);
    Iv lc_sq = isquare(longer);
    Iv sc_sq = isquare(shorter);
    Iv add_term = idiv(isub(lc_sq, sc_sq), ab);
    tighten_lb(add_term, 0.0);

    if (possibly(obt)) {
        Iv lx = iscale(0.5, iadd(add_term, ab));
        Iv sx = iscale(0.5, isub(add_term, ab));
        tighten_lb(sx, 0.0);
        tighten_ub(sx, shorter.ub);
        tighten_ub(lx, longer.ub);
        if (iempty(sx) || iempty(lx)) {
            if (definitely(obt)) t_trap = true;  // collision_angles.cu:59-62
        } else {
            Iv lquot = idiv(lx, longer);
            tighten_ub(lquot, 1.0);
            Iv squot = idiv(sx, shorter);
            tighten_ub(squot, 1.0);
            if (iempty(lquot) || iempty(squot)) {
                if (definitely(obt)) t_trap = true;  // collision_angles.cu:72-75
            } else {
                Iv alpha = iasin(lquot);
                Iv beta = iasin(squot);
                result = isub(alpha, beta);
                tighten_lb(result, 0.0);
            }
        }
    }

    if (!definitely(obt)) {
        Iv lx = iscale(0.5, iadd(ab, add_term));
        Iv sx = iscale(0.5, isub(ab, add_term));
        tighten_lb(sx, 0.0);
        if (iempty(sx)) {
            if (!possibly(obt)) t_trap = true;  // collision_angles.cu:92-101
        } else {
            Iv alpha = iasin(idiv(lx, longer));
            Iv beta = iasin(idiv(sx, shorter));
            tighten_lb(beta, 0.0);
            Iv r = iadd(alpha, beta);
            if (iempty(result))
                result = r;
            else
                ijoin(result, r);
        }
    }
    return result;
}

// collision_angles.cu:119-142
static Iv ca_inner_inner(Iv la, Iv ra, Iv rb) {
    double lb, ub;
    {
        Iv lc = iadd(pt(ra.ub), pt(la.lb));
        Iv sc = iadd(pt(rb.ub), pt(la.lb));
        Iv ab = iadd(pt(ra.ub), pt(rb.ub));
        ub = collision_angle(lc, sc, ab).ub;
    }
    {
        Iv lc = iadd(pt(ra.lb), pt(la.ub));
        Iv sc = iadd(pt(rb.lb), pt(la.ub));
        Iv ab = iadd(pt(ra.lb), pt(rb.lb));
        if (ab.lb <= 0.0)
            lb = 0.0;
        else
            lb = collision_angle(lc, sc, ab).lb;
    }
    return {lb, ub};
}

// collision_angles.cu:144-158 / 175-189: one ordering or the join of both
static Iv ca_ordered(Iv ca, Iv cb, Iv ab) {
    Ub ca_longer = ile(cb, ca);
    if (definitely(ca_longer)) return collision_angle(ca, cb, ab);
    if (definitely(unot(ca_longer))) return collision_angle(cb, ca, ab);
    Iv result = collision_angle(ca, cb, ab);
    ijoin(result, collision_angle(cb, ca, ab));
    return result;
}
static Iv do_outer_inner(Iv la, Iv ra, Iv rb) {
    Iv ca = isub(pt(1.0), ra);
    Iv cb = iadd(la, rb);
    Iv ab = iadd(ra, rb);
    return ca_ordered(ca, cb, ab);
}
static Iv do_inner_outer(Iv la, Iv ra, Iv rb) {
    Iv ca = iadd(la, ra);
    Iv cb = isub(pt(1.0), rb);
    Iv ab = iadd(ra, rb);
    return ca_ordered(ca, cb, ab);
}
// collision_angles.cu:160-173
static Iv ca_outer_inner(Iv la, Iv ra, Iv rb) {
    double lb, ub;
    if (possibly(ile(iscale(2.0, iadd(ra, rb)), isub(pt(1.0), la))))
        lb = 0.0;
    else
        lb = do_outer_inner(la, pt(ra.lb), pt(rb.lb)).lb;
    ub = do_outer_inner(la, pt(ra.ub), pt(rb.ub)).ub;
    return {lb, ub};
}
// collision_angles.cu:191-205
static Iv ca_inner_outer(Iv la, Iv ra, Iv rb) {
    double lb, ub;
    if (possibly(ile(iscale(2.0, iadd(ra, rb)), isub(pt(1.0), la))))
        lb = 0.0;
    else
        lb = do_inner_outer(la, pt(ra.lb), pt(rb.lb)).lb;
    ub = do_inner_outer(la, pt(ra.ub), pt(rb.ub)).ub;
    return {lb, ub};
}
// collision_angles.cu:207-231
static Iv ca_outer_outer(Iv ra, Iv rb) {
    double lb, ub;
    {
        Iv lc = isub(pt(1.0), pt(rb.ub));
        Iv sc = isub(pt(1.0), pt(ra.ub));
        Iv ab = iadd(pt(ra.ub), pt(rb.ub));
        ub = collision_angle(lc, sc, ab).ub;
    }
    {
        Iv lc = isub(pt(1.0), pt(rb.lb));
        Iv sc = isub(pt(1.0), pt(ra.lb));
        Iv ab = iadd(pt(ra.lb), pt(rb.lb));
        if (ab.lb <= 0.0)
            lb = 0.0;
        else
            lb = collision_angle(lc, sc, ab).lb;
    }
    return {lb, ub};
}
// collision_angles.cu:233-238
static Iv semi_outer(Iv r) {
    return {asin_rd(div_rd(r.lb, add_ru(1.0, -r.lb))), asin_ru(div_ru(r.ub, add_rd(1.0, -r.ub)))};
}
// collision_angles.cu:240-246
static Iv semi_inner(Iv la, Iv r) {
    return {asin_rd(div_rd(r.lb, add_ru(la.ub, r.lb))), asin_ru(div_ru(r.ub, add_rd(la.lb, r.ub)))};
}

// lower_bound_radius_single_placement.cu:26-61
static double single_placement(double lb_lambda) {
    const double f = div_ru(kCriticalRatio, kLbPi);
    const double rhs = mul_ru(f, add_ru(1.0, -mul_rd(lb_lambda, lb_lambda)));
    double ub = 0.25, lb = 5.0e-324;
    for (;;) {
        double mid = 0.5 * (lb + ub);
        if (mid <= lb || mid >= ub) return ub;
        double r_sq = mul_rd(mid, mid);
        double q = div_ru(mid, add_rd(1.0, -mid));
        double s = asin_ru(q);
        double lhs = div_rd(r_sq, s);
        if (lhs >= rhs)
            ub = mid;
        else
            lb = mid;
    }
}

// subintervals.hpp:31-42.  On the device nvcc contracts lb + diff*i into one
// FMA; `fused` selects that form (std::fma is correctly rounded, like the GPU's).
static inline Iv subinterval(Iv iv, int i, int n, bool fused) {
    double lb = iv.lb, ub = iv.ub;
    double diff = ub - lb;
    diff /= n;
    double l, u;
    if (fused) {
        l = std::fma(diff, (double)i, lb);
        u = std::fma(diff, (double)(i + 1), lb);
    } else {
        volatile double t1 = diff * i, t2 = diff * (i + 1);
        l = lb + t1;
        u = lb + t2;
    }
    if (i + 1 == n) u = ub;
    return {l, u};
}

// ---------------------------------------------------------------- families
enum Family { START = 0, START_END_2D = 1, START_END_3D = 2, MIDDLE = 3, END_2D = 4, END_3D = 5 };
static inline int family_dims(int fam) { return (fam == START_END_2D || fam == END_2D) ? 3 : 4; }

// start_configuration.cu:58-66 (identical in middle_configuration.cu:66-74, end_configuration.cu:55-63)
static Iv range_r1(Iv la, double single) {
    double ub_lane = iscale(0.5, isub(pt(1.0), la)).ub;
    double lb_lane = iscale(0.25, isub(pt(1.0), la)).lb;
    return {lb_lane, ub_lane < single ? ub_lane : single};
}
static Iv range_r2(int fam, Iv la, Iv r1) {
    if (fam == START_END_2D) {
        // start_configuration.cu:74-77 (compute_r2_range_2d)
        double lb = iscale(0.5, isub(isub(pt(1.0), la), iscale(2.0, r1))).lb;
        return {lb, r1.ub};
    }
    if (fam == END_2D || fam == END_3D) {
        // end_configuration.cu:65-69
        double lb = mul_rd(0.5, add_rd(1.0, -add_ru(la.ub, mul_ru(2.0, r1.ub))));
        if (lb < 0.0) lb = 0.0;
        return {lb, r1.ub};
    }
    // start_configuration.cu:68-71, middle_configuration.cu:76-79
    return {iscale(0.25, isub(pt(1.0), la)).lb, r1.ub};
}
static Iv range_r3(int fam, Iv la, Iv r2) {
    if (fam == START_END_3D) {
        // start_configuration.cu:84-87 (compute_r3_range_3d)
        double lb = iscale(0.5, isub(isub(pt(1.0), la), iscale(2.0, r2))).lb;
        return {lb, r2.ub};
    }
    if (fam == END_3D) {
        // end_configuration.cu:148-152
        double lb = mul_rd(0.5, add_rd(1.0, -add_ru(la.ub, mul_ru(2.0, r2.ub))));
        if (lb < 0.0) lb = 0.0;
        return {lb, r2.ub};
    }
    // start_configuration.cu:79-82, middle_configuration.cu:81-84
    return {iscale(0.25, isub(pt(1.0), la)).lb, r2.ub};
}

// ratio (1 - lambda^2) upper bound, shared by every criterion
static inline double area_ratio_ub(Iv la) { return add_ru(1.0, -mul_rd(la.lb, la.lb)); }
static inline double disk_area_lb(Iv r) { return mul_rd(kLbPi, mul_rd(r.lb, r.lb)); }

// Per-box result.  Sub-criterion k "fails" sets bit k of mask; bit 6 = the
// fit check fired; bit 7 = a reference trap site was reached.
enum : uint8_t { V_PROVED = 0, V_CRITICAL = 1, V_NOFIT = 2, V_EMPTY = 3, V_ERROR = 4 };
enum : uint8_t { M_FIT = 0x40, M_TRAP = 0x80 };
struct Out {
    uint8_t verdict, mask;
    double trace[8][2];  // (lhs, rhs) per sub-criterion; NaN when not evaluated
};
static inline void set_trace(Out& o, int k, double lhs, double rhs) {
    o.trace[k][0] = lhs;
    o.trace[k][1] = rhs;
}

// start_configuration.cu:93-101 (handle_case_1); returns the compared pair
static bool start_case_1(Iv la, Iv r1, Iv r2, Iv a12, double* lhs, double* rhs) {
    double ratio = area_ratio_ub(la);
    double a1 = disk_area_lb(r1), a2 = disk_area_lb(r2);
    Iv a = iadd(semi_outer(r1), a12);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    *lhs = add_rd(a1, mul_rd(0.5, a2));
    *rhs = mul_ru(kCriticalRatio, used);
    return *lhs >= *rhs;
}
// start_configuration.cu:103-111 (handle_case_2)
static bool start_case_2(Iv la, Iv r1, Iv r2, Iv r3, Iv a13, double* lhs, double* rhs) {
    double ratio = area_ratio_ub(la);
    double a1 = disk_area_lb(r1), a2 = disk_area_lb(r2), a3 = disk_area_lb(r3);
    Iv a = iadd(semi_outer(r1), a13);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    *lhs = add_rd(add_rd(a1, a2), mul_rd(0.5, a3));
    *rhs = mul_ru(kCriticalRatio, used);
    return *lhs >= *rhs;
}
// start_configuration.cu:169-188 (handle_2d_case)
static bool start_end_2d_case(Iv la, Iv r1, Iv r2, double* lhs, double* rhs) {
    Iv a1 = semi_outer(r1);
    Iv a2 = semi_inner(la, r2);
    Iv a12 = ca_outer_inner(la, r1, r2);
    Iv total = iadd(iadd(a1, a2), a12);
    Iv reuse = isub(iadd(a12, a2), a1);
    tighten_lb(reuse, 0.0);
    double ratio = area_ratio_ub(la);
    double used = mul_ru(ratio, mul_ru(0.5, total.ub));
    Iv rho = isub(pt(1.0), isquare(iadd(la, iscale(2.0, r2))));
    tighten_lb(rho, 0.0);
    double reusable = mul_rd(mul_rd(0.5, reuse.lb), rho.lb);
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
    *lhs = add_rd(ar2, ar1);
    *rhs = mul_ru(kCriticalRatio, add_ru(used, -reusable));
    return *lhs >= *rhs;
}
// start_configuration.cu:227-265 (handle_3d_case).  Note the reference computes
// a13 from (r1, r2) here (start_configuration.cu:232); restated as written.
static bool start_end_3d_case(Iv la, Iv r1, Iv r2, Iv r3, double* lhs, double* rhs) {
    Iv a1 = semi_outer(r1);
    Iv a2 = semi_inner(la, r2);
    Iv a3 = semi_outer(r3);
    Iv a12 = ca_outer_inner(la, r1, r2);
    Iv a13 = ca_outer_outer(r1, r2);
    Iv a23 = ca_inner_outer(la, r2, r3);
    Iv b123 = iadd(a12, a23);
    Iv b13{a13.lb < b123.lb ? b123.lb : a13.lb, a13.ub < b123.ub ? b123.ub : a13.ub};
    Iv a123 = iadd(iadd(a1, b13), a3);
    Iv a122 = iadd(iadd(a1, a12), a2);
    Iv a{a123.lb < a122.lb ? a122.lb : a123.lb, a123.ub < a122.ub ? a122.ub : a123.ub};
    double reuse_angle = isub(a, a122).lb;
    if (reuse_angle < 0.0) reuse_angle = 0.0;
    double outer_rad = add_rd(1.0, -mul_ru(2.0, r3.ub));
    double outer_sq = mul_rd(outer_rad, outer_rad);
    double inner_rad = la.ub;
    double inner_sq = mul_ru(inner_rad, inner_rad);
    double reused = mul_rd(mul_rd(0.5, reuse_angle), add_rd(outer_sq, -inner_sq));
    if (reused < 0.0) reused = 0.0;
    double ratio = area_ratio_ub(la);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    used = add_ru(used, -reused);
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2), ar3 = disk_area_lb(r3);
    *lhs = add_rd(ar1, add_rd(ar2, ar3));
    *rhs = mul_ru(kCriticalRatio, used);
    return *lhs >= *rhs;
}
// middle_configuration.cu:86-119 / 121-154: two guarded sub-checks; a
// sub-check fails when lb_disk_area < critical_ratio * ub_area_used.
static void middle_case(Iv la, Iv r1, Iv r2, Iv r3, Iv c12, Iv c13, Iv c23, Out& o, int k0) {
    double ratio = area_ratio_ub(la);
    Ub case_a = ige(iadd(c12, c23), c13);
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
    if (possibly(case_a)) {
        double used = mul_ru(ratio, mul_ru(0.5, c12.ub));
        double lhs = mul_rd(0.5, add_rd(ar1, ar2));
        double rhs = mul_ru(kCriticalRatio, used);
        set_trace(o, k0, lhs, rhs);
        if (lhs < rhs) {
            o.mask |= (uint8_t)(1u << k0);
            if (t_decide) return;
        }
    }
    if (possibly(unot(case_a))) {
        double used = mul_ru(ratio, mul_ru(0.5, c13.ub));
        double ar3 = disk_area_lb(r3);
        double lhs = add_rd(mul_rd(0.5, add_rd(ar1, ar3)), ar2);
        double rhs = mul_ru(kCriticalRatio, used);
        set_trace(o, k0 + 1, lhs, rhs);
        if (lhs < rhs) o.mask |= (uint8_t)(1u << (k0 + 1));
    }
}
// end_configuration.cu:71-85 (handle_inner_outer_2d)
static bool end_inner_outer_2d(Iv la, Iv r1, Iv r2, double* lhs, double* rhs) {
    Iv a = iadd(ca_inner_outer(la, r1, r2), semi_outer(r2));
    double ratio = area_ratio_ub(la);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    Iv rho = isub(isquare(isub(pt(1.0), iscale(2.0, r2))), isquare(la));
    tighten_lb(rho, 0.0);
    double alpha = isub(a, semi_inner(la, r1)).lb;
    double reusable = mul_rd(mul_rd(0.5, alpha), rho.lb);
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
    *lhs = add_rd(ar2, mul_rd(0.5, ar1));
    *rhs = mul_ru(kCriticalRatio, add_ru(used, -reusable));
    return *lhs >= *rhs;
}
// end_configuration.cu:87-101 (handle_outer_inner_2d)
static bool end_outer_inner_2d(Iv la, Iv r1, Iv r2, double* lhs, double* rhs) {
    Iv a = iadd(ca_outer_inner(la, r1, r2), semi_inner(la, r2));
    double ratio = area_ratio_ub(la);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    Iv rho = isub(pt(1.0), isquare(iadd(la, iscale(2.0, r2))));
    tighten_lb(rho, 0.0);
    double alpha = isub(a, semi_outer(r1)).lb;
    double reusable = mul_rd(mul_rd(0.5, alpha), rho.lb);
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
    *lhs = add_rd(ar2, mul_rd(0.5, ar1));
    *rhs = mul_ru(kCriticalRatio, add_ru(used, -reusable));
    return *lhs >= *rhs;
}
// end_configuration.cu:154-181 (handle_r1_inner_3d) and 183-210
// (handle_r1_outer_3d).  Returns -1 when the early "definitely" exit applies.
static int end_3d_case(bool r1_inner, Iv la, Iv r1, Iv r2, Iv r3, double* lhs, double* rhs) {
    Iv a12, a23, a13;
    if (r1_inner) {
        a12 = ca_inner_outer(la, r1, r2);
        a23 = ca_outer_inner(la, r2, r3);
        a13 = ca_inner_inner(la, r1, r3);
    } else {
        a12 = ca_outer_inner(la, r1, r2);
        a23 = ca_inner_outer(la, r2, r3);
        a13 = ca_outer_outer(r1, r3);
    }
    if (definitely(ige(iadd(a12, a23), a13))) return -1;
    Iv a3 = r1_inner ? semi_inner(la, r3) : semi_outer(r3);
    Iv a = iadd(a13, a3);
    Iv a2 = r1_inner ? semi_outer(r2) : semi_inner(la, r2);
    Iv reusable_alpha = isub(a, iadd(a12, a2));
    Iv rho = r1_inner ? isub(pt(1.0), isquare(iadd(la, iscale(2.0, r3))))
                      : isub(isquare(isub(pt(1.0), iscale(2.0, r3))), isquare(la));
    tighten_lb(rho, 0.0);
    double reusable = mul_rd(mul_rd(0.5, reusable_alpha.lb), rho.lb);
    double ratio = area_ratio_ub(la);
    double used = mul_ru(ratio, mul_ru(0.5, a.ub));
    double ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2), ar3 = disk_area_lb(r3);
    *lhs = add_rd(add_rd(ar2, ar3), mul_rd(0.5, ar1));
    *rhs = mul_ru(kCriticalRatio, add_ru(used, -reusable));
    return *lhs >= *rhs ? 1 : 0;
}

// The body of each family kernel's innermost loop, for one raw box
// (la, r1_, r2_[, r3]): the tightening, the fit check, and every criterion.
// start_configuration.cu:126-162, 200-212, 277-295; middle_configuration.cu:166-201;
// end_configuration.cu:109-144, 223-265.  Every sub-criterion is evaluated
// (the reference kernel stops at the first failure; the mask records all).
// A box with an empty axis after tightening is EMPTY (end_configuration.cu:222-234
// skips such boxes; the other families' lattices never produce them).
static void eval_box(int fam, const double* lo, const double* hi, Out& o) {
    o.verdict = V_PROVED;
    o.mask = 0;
    for (int k = 0; k < 8; ++k) o.trace[k][0] = o.trace[k][1] = NAN;
    t_trap = false;
    const int dims = family_dims(fam);
    Iv la{lo[0], hi[0]}, r1{lo[1], hi[1]}, r2{lo[2], hi[2]}, r3{0.0, 0.0};
    if (dims == 4) {
        r3 = {lo[3], hi[3]};
        tighten_lb(r2, r3.lb);
    }
    tighten_lb(r1, r2.lb);
    if (iempty(la) || iempty(r1) || iempty(r2) || (dims == 4 && iempty(r3))) {
        o.verdict = V_EMPTY;
        return;
    }
    bool fit_fires = mul_ru(2.0, r1.ub) >= add_rd(1.0, -la.ub);
    double lhs, rhs;
    switch (fam) {
    case START: {
        if (fit_fires) o.mask |= M_FIT;
        Iv a12 = ca_outer_inner(la, r1, r2);
        Iv a13 = ca_outer_outer(r1, r3);
        Iv a23 = ca_inner_outer(la, r2, r3);
        Ub case1 = igt(iadd(a12, a23), a13);
        if (possibly(case1)) {
            if (!start_case_1(la, r1, r2, a12, &lhs, &rhs)) o.mask |= 1;
            set_trace(o, 0, lhs, rhs);
            if (t_decide && (o.mask & 1)) break;
        }
        if (possibly(unot(case1))) {
            if (!start_case_2(la, r1, r2, r3, a13, &lhs, &rhs)) o.mask |= 2;
            set_trace(o, 1, lhs, rhs);
        }
        break;
    }
    case START_END_2D:
        if (!start_end_2d_case(la, r1, r2, &lhs, &rhs)) o.mask |= 1;
        set_trace(o, 0, lhs, rhs);
        break;
    case START_END_3D:
        if (!start_end_3d_case(la, r1, r2, r3, &lhs, &rhs)) o.mask |= 1;
        set_trace(o, 0, lhs, rhs);
        break;
    case MIDDLE: {
        if (fit_fires) o.mask |= M_FIT;
        if (t_decide && fit_fires) break;
        Iv c12 = ca_inner_outer(la, r1, r2), c13 = ca_inner_inner(la, r1, r3), c23 = ca_outer_inner(la, r2, r3);
        middle_case(la, r1, r2, r3, c12, c13, c23, o, 0);
        if (t_decide && (o.mask & 3)) break;
        Iv d12 = ca_outer_inner(la, r1, r2), d13 = ca_outer_outer(r1, r3), d23 = ca_inner_outer(la, r2, r3);
        middle_case(la, r1, r2, r3, d12, d13, d23, o, 2);
        break;
    }
    case END_2D:
        if (fit_fires) o.mask |= M_FIT;
        if (t_decide && fit_fires) break;
        if (!end_inner_outer_2d(la, r1, r2, &lhs, &rhs)) o.mask |= 1;
        set_trace(o, 0, lhs, rhs);
        if (t_decide && (o.mask & 1)) break;
        if (!end_outer_inner_2d(la, r1, r2, &lhs, &rhs)) o.mask |= 2;
        set_trace(o, 1, lhs, rhs);
        break;
    case END_3D: {
        if (fit_fires) o.mask |= M_FIT;
        if (t_decide && fit_fires) break;
        for (int k = 0; k < 2; ++k) {
            int r = end_3d_case(k == 0, la, r1, r2, r3, &lhs, &rhs);
            if (r >= 0) set_trace(o, k, lhs, rhs);
            if (r == 0) o.mask |= (uint8_t)(1u << k);
            if (t_decide && r == 0) break;
        }
        break;
    }
    }
    if (t_trap) o.mask |= M_TRAP;
    if (o.mask & M_TRAP)
        o.verdict = V_ERROR;
    else if ((o.mask & M_FIT) && fam != START)
        o.verdict = V_NOFIT;
    else if (o.mask & 0x3F)
        o.verdict = V_CRITICAL;
    else
        o.verdict = V_PROVED;
}

// ---------------------------------------------------------------- lattice
// The box at lattice coordinates (i_la, i_r1, i_r2[, i_r3]) of a family kernel's
// nested loops (e.g. middle_configuration.cu:157-168): each axis is the i-th
// subinterval of its dependent range.  `single` is the single-placement bound
// of la.lb (compute_r1_range).
struct LatticeSpec {
    int fam;
    int n[4];
    Iv outer;
    bool fused;
};
// Returns false for boxes the kernel never visits: end_configuration.cu:225-227
// skips the r3 loop when the r3 range is empty.
static bool lattice_box(const LatticeSpec& s, const int* ix, double single, double* lo, double* hi) {
    Iv la = subinterval(s.outer, ix[0], s.n[0], s.fused);
    Iv r1 = subinterval(range_r1(la, single), ix[1], s.n[1], s.fused);
    Iv r2 = subinterval(range_r2(s.fam, la, r1), ix[2], s.n[2], s.fused);
    lo[0] = la.lb; hi[0] = la.ub;
    lo[1] = r1.lb; hi[1] = r1.ub;
    lo[2] = r2.lb; hi[2] = r2.ub;
    if (family_dims(s.fam) == 4) {
        Iv r3r = range_r3(s.fam, la, r2);
        Iv r3 = subinterval(r3r, ix[3], s.n[3], s.fused);
        lo[3] = r3.lb; hi[3] = r3.ub;
        if (s.fam == END_3D && iempty(r3r)) return false;
    }
    return true;
}
static inline void unravel(const LatticeSpec& s, int64_t idx, int* ix) {
    int dims = family_dims(s.fam);
    for (int d = dims - 1; d >= 0; --d) {
        ix[d] = (int)(idx % s.n[d]);
        idx /= s.n[d];
    }
}

// ---------------------------------------------------------------- threading
template <class F>
static void parallel_for(int64_t n, int nthreads, F&& f) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads < 1) nthreads = 1;
    if (n < 256 || nthreads == 1) {
        f(0, n, 0);
        return;
    }
    if ((int64_t)nthreads > n) nthreads = (int)n;
    std::atomic<int64_t> next{0};
    const int64_t chunk = 1024;
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
        pool.emplace_back([&, t] {
            for (;;) {
                int64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                int64_t e = b + chunk < n ? b + chunk : n;
                f(b, e, t);
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------- C API
extern "C" {

int orc_family_dims(int fam) { return family_dims(fam); }

// Evaluate n raw boxes (SoA: lo[d*stride + i]).  trace may be NULL; else
// n*8*2 doubles (per box, per sub-criterion: lhs, rhs).
int orc_eval_boxes(int fam, const double* lo, const double* hi, int64_t n, int64_t stride,
                   uint8_t* verdict, uint8_t* mask, double* trace, int nthreads) {
    if (fam < 0 || fam > 5 || n < 0) return 1;
    const int dims = family_dims(fam);
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        double l[4], h[4];
        Out o;
        for (int64_t i = b; i < e; ++i) {
            for (int d = 0; d < dims; ++d) {
                l[d] = lo[d * stride + i];
                h[d] = hi[d * stride + i];
            }
            eval_box(fam, l, h, o);
            verdict[i] = o.verdict;
            mask[i] = o.mask;
            if (trace) std::memcpy(trace + i * 16, o.trace, sizeof(o.trace));
        }
    });
    return 0;
}

// The box refinement of the device engine with the uniform split (every axis
// bisected), restated on the CPU for the boxes below a sample of lattice seed
// boxes, on the reference kernel's own evaluation path (stop at the first
// failing sub-check and handle, and at a firing fit check where the kernel
// traps).  A box that is neither proved nor empty is unresolved at max_depth,
// else its 2^dims children (midpoints rounded to nearest) are intersected with
// the dependent ranges of their own lambda interval (single-placement bound from
// the same 2^16-point lambda grid as the device: the value at the largest grid
// point <= lambda.lb) and evaluated in turn; children with an empty range are
// dropped (clipped).  out[0..4]: verdict counts, out[5] unresolved, out[6]
// clipped; per_depth[d] evaluated boxes at depth d < 16; ops[4 d + k]
// primitive counts (add, mul, div, asin) at depth d < 16 (may be NULL).
struct SingleGrid {
    std::vector<double> t, v;
    double h = 0.0;
};
static const SingleGrid& single_grid() {
    static SingleGrid g = [] {
        SingleGrid s;
        const int n = 1 << 16;
        s.h = (kLambdaMax - kLambdaMin) / (n - 1);
        s.t.resize(n);
        s.v.resize(n);
        parallel_for(n, 0, [&](int64_t b, int64_t e, int) {
            for (int64_t i = b; i < e; ++i) {
                s.t[i] = std::fma((double)i, s.h, kLambdaMin);
                s.v[i] = single_placement(s.t[i]);
            }
        });
        return s;
    }();
    return g;
}
static double single_upper(const SingleGrid& g, double la_lo) {
    if (!(la_lo >= g.t[0])) return 0.25;
    int64_t i = (int64_t)((la_lo - g.t[0]) / g.h);
    const int64_t n = (int64_t)g.t.size();
    if (i >= n) i = n - 1;
    while (i > 0 && g.t[i] > la_lo) --i;
    while (i + 1 < n && g.t[i + 1] <= la_lo) ++i;
    return g.v[i];
}
static bool clip_child(int fam, const SingleGrid& g, double* lo, double* hi) {
    const Iv la{lo[0], hi[0]};
    const Iv r1r = range_r1(la, single_upper(g, la.lb));
    if (lo[1] < r1r.lb) lo[1] = r1r.lb;
    if (r1r.ub < hi[1]) hi[1] = r1r.ub;
    if (lo[1] > hi[1]) return false;
    const Iv r2r = range_r2(fam, la, Iv{lo[1], hi[1]});
    if (lo[2] < r2r.lb) lo[2] = r2r.lb;
    if (r2r.ub < hi[2]) hi[2] = r2r.ub;
    if (lo[2] > hi[2]) return false;
    if (family_dims(fam) == 4) {
        const Iv r3r = range_r3(fam, la, Iv{lo[2], hi[2]});
        if (lo[3] < r3r.lb) lo[3] = r3r.lb;
        if (r3r.ub < hi[3]) hi[3] = r3r.ub;
        if (lo[3] > hi[3]) return false;
    }
    return true;
}
struct RefineTally {
    int64_t out[7] = {0, 0, 0, 0, 0, 0, 0};
    int64_t per_depth[16] = {0};
    OpCount ops[16] = {};
};
static void refine_box(int fam, const SingleGrid& g, const double* lo, const double* hi, int depth, int max_depth,
                       RefineTally& t) {
    const int dims = family_dims(fam);
    const int dd = depth < 16 ? depth : 15;
    Out o;
    OpCount c{0, 0, 0, 0};
    t_count = &c;
    eval_box(fam, lo, hi, o);
    t_count = nullptr;
    t.ops[dd].add += c.add;
    t.ops[dd].mul += c.mul;
    t.ops[dd].div += c.div;
    t.ops[dd].asin += c.asin;
    t.out[o.verdict]++;
    t.per_depth[dd]++;
    if (o.verdict == V_PROVED || o.verdict == V_EMPTY) return;
    if (depth >= max_depth) {
        t.out[5]++;
        return;
    }
    double mid[4];
    for (int d = 0; d < dims; ++d) mid[d] = 0.5 * (lo[d] + hi[d]);
    for (int k = 0; k < (1 << dims); ++k) {
        double cl[4], ch[4];
        for (int d = 0; d < dims; ++d) {
            cl[d] = ((k >> d) & 1) ? mid[d] : lo[d];
            ch[d] = ((k >> d) & 1) ? hi[d] : mid[d];
        }
        if (!clip_child(fam, g, cl, ch)) {
            t.out[6]++;
            continue;
        }
        refine_box(fam, g, cl, ch, depth + 1, max_depth, t);
    }
}

// Count the primitive operations of the evaluation of n boxes.
// counts[0..3] = add/sub, mul, div, asin (summed over the boxes).  decide = 0:
// every sub-criterion (FULL); decide = 1: the reference kernel's own path, which
// stops at the first failing sub-check / handle and at a firing fit check.
int orc_count_ops_mode(int fam, const double* lo, const double* hi, int64_t n, int64_t stride, int decide,
                       uint64_t* counts) {
    if (fam < 0 || fam > 5 || n < 0) return 1;
    const int dims = family_dims(fam);
    OpCount c{0, 0, 0, 0};
    t_count = &c;
    t_decide = decide != 0;
    double l[4], h[4];
    Out o;
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dims; ++d) {
            l[d] = lo[d * stride + i];
            h[d] = hi[d * stride + i];
        }
        eval_box(fam, l, h, o);
    }
    t_count = nullptr;
    t_decide = false;
    counts[0] = c.add;
    counts[1] = c.mul;
    counts[2] = c.div;
    counts[3] = c.asin;
    return 0;
}
int orc_count_ops(int fam, const double* lo, const double* hi, int64_t n, int64_t stride, uint64_t* counts) {
    return orc_count_ops_mode(fam, lo, hi, n, stride, 0, counts);
}

// The uniform refinement below the lattice seed boxes idx[0..n) of a family
// lattice (see refine_box), over nthreads host threads (0 = all).
int orc_refine_sample(int fam, double outer_lb, double outer_ub, const int32_t* sizes, const int64_t* idx, int64_t n,
                      int max_depth, int64_t* out, int64_t* per_depth, uint64_t* ops, int nthreads) {
    if (fam < 0 || fam > 5 || n < 0 || max_depth < 0 || max_depth > 15 || !out) return 1;
    LatticeSpec s{fam, {sizes[0], sizes[1], sizes[2], family_dims(fam) == 4 ? sizes[3] : 1},
                  {outer_lb, outer_ub}, true};
    const SingleGrid& g = single_grid();
    int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    std::vector<RefineTally> tally((size_t)nt);
    // the lattice kernels' own single-placement bound per lambda slab (exact, as the seed)
    std::vector<double> single(s.n[0], -1.0);
    std::vector<std::once_flag> once(s.n[0]);
    const int dims = family_dims(fam);
    // small work items: one seed box each (the trees below seeds differ widely in size)
    std::atomic<int64_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) {
        pool.emplace_back([&, t] {
            t_decide = true;
            int ix[4] = {0, 0, 0, 0};
            double l[4], h[4];
            for (;;) {
                const int64_t i = next.fetch_add(1);
                if (i >= n) break;
                unravel(s, idx[i], ix);
                std::call_once(once[ix[0]], [&] {
                    single[ix[0]] = single_placement(subinterval(s.outer, ix[0], s.n[0], s.fused).lb);
                });
                if (!lattice_box(s, ix, single[ix[0]], l, h)) {
                    tally[t].out[6]++;
                    continue;
                }
                refine_box(fam, g, l, h, 0, max_depth, tally[t]);
            }
            t_decide = false;
        });
    }
    for (auto& th : pool) th.join();
    for (int k = 0; k < 7; ++k) out[k] = 0;
    for (int d = 0; d < 16; ++d) {
        if (per_depth) per_depth[d] = 0;
        if (ops) ops[4 * d] = ops[4 * d + 1] = ops[4 * d + 2] = ops[4 * d + 3] = 0;
    }
    for (const auto& ta : tally) {
        for (int k = 0; k < 7; ++k) out[k] += ta.out[k];
        for (int d = 0; d < 16; ++d) {
            if (per_depth) per_depth[d] += ta.per_depth[d];
            if (ops) {
                ops[4 * d] += ta.ops[d].add;
                ops[4 * d + 1] += ta.ops[d].mul;
                ops[4 * d + 2] += ta.ops[d].div;
                ops[4 * d + 3] += ta.ops[d].asin;
            }
        }
    }
    (void)dims;
    return 0;
}

double orc_single_placement(double lb_lambda) { return single_placement(lb_lambda); }

void orc_asin_pad(const double* x, int64_t n, double* rd, double* ru) {
    for (int64_t i = 0; i < n; ++i) {
        rd[i] = asin_rd(x[i]);
        ru[i] = asin_ru(x[i]);
    }
}

// Directed-rounding primitives, for the tests that check them against <cfenv>.
// op: 0 add, 1 mul, 2 div; up: 0 = toward -inf, 1 = toward +inf.
void orc_round_op(int op, int up, const double* a, const double* b, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        if (op == 0)
            out[i] = add_dir(a[i], b[i], up != 0);
        else if (op == 1)
            out[i] = mul_dir(a[i], b[i], up != 0);
        else
            out[i] = div_dir(a[i], b[i], up != 0);
    }
}
void orc_round_op_fenv(int op, int up, const double* a, const double* b, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = slow_op(op, up != 0, a[i], b[i]);
}

// Primitive geometry on interval arrays (in[k*n + i] holds argument k as lb/ub
// pairs: in[(2k)*n + i] = lb, in[(2k+1)*n + i] = ub).  kind: 0 inner_inner(la,ra,rb),
// 1 outer_inner(la,ra,rb), 2 inner_outer(la,ra,rb), 3 outer_outer(ra,rb),
// 4 semicircle_outer(r), 5 semicircle_inner(la,r).  out: lb[i], ub[n+i]; trap[i].
int orc_primitive(int kind, const double* in, int64_t n, double* out, uint8_t* trap) {
    for (int64_t i = 0; i < n; ++i) {
        Iv a0{in[0 * n + i], in[1 * n + i]}, a1{in[2 * n + i], in[3 * n + i]};
        Iv a2{0, 0};
        if (kind <= 2) a2 = {in[4 * n + i], in[5 * n + i]};
        t_trap = false;
        Iv r;
        switch (kind) {
        case 0: r = ca_inner_inner(a0, a1, a2); break;
        case 1: r = ca_outer_inner(a0, a1, a2); break;
        case 2: r = ca_inner_outer(a0, a1, a2); break;
        case 3: r = ca_outer_outer(a0, a1); break;
        case 4: r = semi_outer(a0); break;
        case 5: r = semi_inner(a0, a1); break;
        default: return 1;
        }
        out[i] = r.lb;
        out[n + i] = r.ub;
        if (trap) trap[i] = t_trap ? 1 : 0;
    }
    return 0;
}

// Boxes of a family lattice at the given linear indices (r3 fastest).
int orc_lattice_boxes(int fam, double outer_lb, double outer_ub, const int32_t* sizes, int fused,
                      const int64_t* idx, int64_t n, double* lo, double* hi, int64_t stride, int nthreads) {
    if (fam < 0 || fam > 5) return 1;
    LatticeSpec s{fam, {sizes[0], sizes[1], sizes[2], family_dims(fam) == 4 ? sizes[3] : 1},
                  {outer_lb, outer_ub}, fused != 0};
    const int dims = family_dims(fam);
    // single-placement bounds per lambda slab
    std::vector<double> single(s.n[0]);
    parallel_for(s.n[0], nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) single[i] = single_placement(subinterval(s.outer, (int)i, s.n[0], s.fused).lb);
    });
    parallel_for(n, nthreads, [&](int64_t b, int64_t e, int) {
        int ix[4] = {0, 0, 0, 0};
        double l[4], h[4];
        for (int64_t i = b; i < e; ++i) {
            unravel(s, idx[i], ix);
            lattice_box(s, ix, single[ix[0]], l, h);
            for (int d = 0; d < dims; ++d) {
                lo[d * stride + i] = l[d];
                hi[d * stride + i] = h[d];
            }
        }
    });
    return 0;
}

// Evaluate a whole lattice and histogram the verdicts: hist[v] counts verdict v
// (0..4); first_critical_la = min la.lb over boxes with a failed sub-criterion
// (the value the reference's kernels reduce with Atomic_ordered_double::store_min,
// atomic_float.hpp:45-47), or +inf when there is none.
int orc_eval_lattice(int fam, double outer_lb, double outer_ub, const int32_t* sizes, int fused,
                     int64_t* hist, double* first_critical_la, int nthreads) {
    if (fam < 0 || fam > 5) return 1;
    LatticeSpec s{fam, {sizes[0], sizes[1], sizes[2], family_dims(fam) == 4 ? sizes[3] : 1},
                  {outer_lb, outer_ub}, fused != 0};
    int64_t total = 1;
    for (int d = 0; d < family_dims(fam); ++d) total *= s.n[d];
    std::vector<double> single(s.n[0]);
    parallel_for(s.n[0], nthreads, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) single[i] = single_placement(subinterval(s.outer, (int)i, s.n[0], s.fused).lb);
    });
    int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    std::vector<int64_t> h((size_t)nt * 5, 0);
    std::vector<double> fc((size_t)nt, INFINITY);
    parallel_for(total, nt, [&](int64_t b, int64_t e, int t) {
        int ix[4] = {0, 0, 0, 0};
        double l[4], hh[4];
        Out o;
        for (int64_t i = b; i < e; ++i) {
            unravel(s, i, ix);
            if (!lattice_box(s, ix, single[ix[0]], l, hh)) {
                h[(size_t)t * 5 + V_EMPTY]++;
                continue;
            }
            eval_box(fam, l, hh, o);
            h[(size_t)t * 5 + o.verdict]++;
            if ((o.mask & 0x3F) && l[0] < fc[t]) fc[t] = l[0];
        }
    });
    for (int v = 0; v < 5; ++v) {
        hist[v] = 0;
        for (int t = 0; t < nt; ++t) hist[v] += h[(size_t)t * 5 + v];
    }
    double m = INFINITY;
    for (int t = 0; t < nt; ++t) m = fc[t] < m ? fc[t] : m;
    *first_critical_la = m;
    return 0;
}

// The reference's lambda refinement loop (run_kernel.cuh:61-132) over a family
// lattice of the given sizes: a min-queue of lambda intervals keyed on lb; each
// step evaluates the lattice over the popped interval and, when a box fails,
// continues on [first, ub] or splits at 0.5*(first+ub).  Records each step's
// (la_lb, la_ub, first) in steps[3*k..] (up to max_steps).  Returns the number
// of steps taken; *proved = 1 when the queue emptied within max_steps.
int64_t orc_reference_loop(int fam, const int32_t* sizes, int fused, int64_t max_steps, double* steps,
                           int* proved, int nthreads) {
    struct Cmp {
        bool operator()(const Iv& a, const Iv& b) const { return a.lb > b.lb; }
    };
    std::priority_queue<Iv, std::vector<Iv>, Cmp> q;
    q.push({kLambdaMin, kLambdaMax});
    int64_t k = 0;
    *proved = 0;
    while (!q.empty()) {
        if (k >= max_steps) return k;
        Iv cur = q.top();
        q.pop();
        int64_t hist[5];
        double fp;
        orc_eval_lattice(fam, cur.lb, cur.ub, sizes, fused, hist, &fp, nthreads);
        steps[3 * k + 0] = cur.lb;
        steps[3 * k + 1] = cur.ub;
        steps[3 * k + 2] = fp;
        ++k;
        if (fp != INFINITY) {
            double width_before = cur.ub - cur.lb;
            double width_after = cur.ub - fp;
            if (width_before >= 2 * width_after) {
                q.push({fp, cur.ub});
            } else {
                double mid = 0.5 * (fp + cur.ub);
                if (fp < mid) q.push({fp, mid});
                if (mid <= cur.ub) q.push({mid, cur.ub});
            }
        }
    }
    *proved = 1;
    return k;
}

}  // extern "C"
