// FP32 pre-pass: a certified shadow of the FP64 evaluation.
//
// Every FP64 value v that the FP64 evaluation (cp_fp64.cuh, cp_families.cuh)
// computes is carried here as an FP32 enclosure E = [l, u] with l <= v <= u:
//   * a directed FP64 sum / product / quotient of enclosed operands is enclosed
//     by the FP32 interval operation rounded outward (__fadd_rd/ru, __fmul_rd/ru,
//     __fdiv_rd/ru), because rd32(x) <= rd64(x) <= x <= ru64(x) <= ru32(x);
//   * the FP64 outward-padded asin (5 steps around CUDA's asin) is enclosed by
//     CUDA's asinf padded kAsinfSteps single-precision steps outward (asinf's
//     documented error is 2 ulp; one single ulp spans 2^29 double ulps);
//   * a comparison that only selects the larger / smaller of two values
//     (tighten_lb/ub, joins, max/min) needs no decision: the enclosure of the
//     FP64 result is the max / min of the enclosures;
//   * every other comparison the FP64 code branches on is decided from the
//     enclosures only when they certify its outcome; otherwise `ok` is cleared
//     and the box is left to the FP64 evaluation.
// When `ok` survives, the shadow followed exactly the FP64 control flow, so the
// verdict it reports is the FP64 DECIDE-mode verdict: FP32 decides a box only
// when that verdict is certain, and every bound near a threshold (within the
// FP32 enclosure width, ~1e-6 relative) goes to FP64.  No trap site is followed:
// a certified trap event also hands the box to FP64.
#pragma once
#include "cp_families.cuh"

namespace cpb {

enum PrefilterResult { PF_UNDECIDED = 0, PF_PROVED = 1, PF_EMPTY = 2, PF_CRITICAL = 3, PF_NOFIT = 4 };

namespace f32 {

constexpr int kAsinfSteps = 8;

struct E {
    float l, u;
};

__device__ __forceinline__ E ec(double x) { return {__double2float_rd(x), __double2float_ru(x)}; }
__device__ __forceinline__ E ek(float c) { return {c, c}; }
__device__ __forceinline__ E eadd(E a, E b) { return {__fadd_rd(a.l, b.l), __fadd_ru(a.u, b.u)}; }
__device__ __forceinline__ E eneg(E a) { return {-a.u, -a.l}; }
__device__ __forceinline__ E esub(E a, E b) { return {__fadd_rd(a.l, -b.u), __fadd_ru(a.u, -b.l)}; }
__device__ __forceinline__ E emul(E a, E b) {
    if (a.l >= 0.f && b.l >= 0.f) return {__fmul_rd(a.l, b.l), __fmul_ru(a.u, b.u)};
    const float p1 = __fmul_rd(a.l, b.l), p2 = __fmul_rd(a.l, b.u), p3 = __fmul_rd(a.u, b.l), p4 = __fmul_rd(a.u, b.u);
    const float q1 = __fmul_ru(a.l, b.l), q2 = __fmul_ru(a.l, b.u), q3 = __fmul_ru(a.u, b.l), q4 = __fmul_ru(a.u, b.u);
    return {fminf(fminf(p1, p2), fminf(p3, p4)), fmaxf(fmaxf(q1, q2), fmaxf(q3, q4))};
}
// a / b rounded down (UP = false) or up, bit-identical to __fdiv_rd / __fdiv_ru.
// For |a|, |b| in [2^-60, 2^61): y = rcp.approx(b) (relative error ~2^-23),
// q0 = a*y, then one correction q = q0 + (a - q0*b)*y leaves |q - a/b| far
// below an ulp of q plus half an ulp, so q is faithful; the remainder
// r = a - q*b (one FMA) is then nonzero exactly when a/b != q and keeps its
// sign (|r| >= 2^-107, no underflow), which picks the directed result among q
// and its neighbour.  Other operands (zeros, subnormals, large exponents,
// infinities, NaN) use the IEEE intrinsics.  One shared (not inlined) copy per
// direction keeps the level kernels within the instruction caches.
__device__ __forceinline__ bool fdiv_in_range(float a, float b) {
    const unsigned ea = (__float_as_uint(a) >> 23) & 0xffu, eb = (__float_as_uint(b) >> 23) & 0xffu;
    return (ea - 67u) <= 120u && (eb - 67u) <= 120u;
}
__device__ __forceinline__ float fnext_up(float q) {  // q finite, normal, nonzero
    const int b = __float_as_int(q);
    return __int_as_float(q > 0.f ? b + 1 : b - 1);
}
__device__ __forceinline__ float fnext_down(float q) {
    const int b = __float_as_int(q);
    return __int_as_float(q > 0.f ? b - 1 : b + 1);
}
template <bool UP>
__device__ __forceinline__ float fdiv_dir_inline(float a, float b) {
    if (!fdiv_in_range(a, b)) return UP ? __fdiv_ru(a, b) : __fdiv_rd(a, b);
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    float q = __fmul_rn(a, y);
    q = __fmaf_rn(__fmaf_rn(-q, b, a), y, q);
    const float r = __fmaf_rn(-q, b, a);
    if (r == 0.f) return q;
    const bool above = (r > 0.f) != (b < 0.f);  // a/b > q
    if (UP) return above ? fnext_up(q) : q;
    return above ? q : fnext_down(q);
}
static __device__ __noinline__ float fdiv_rd(float a, float b) { return fdiv_dir_inline<false>(a, b); }
static __device__ __noinline__ float fdiv_ru(float a, float b) { return fdiv_dir_inline<true>(a, b); }

// enclosure of a/b; the divisor enclosure must exclude 0
__device__ __forceinline__ E ediv(E a, E b, bool& ok) {
    if (b.l > 0.f) {
        if (a.l >= 0.f) return {fdiv_rd(a.l, b.u), fdiv_ru(a.u, b.l)};
        if (a.u <= 0.f) return {fdiv_rd(a.l, b.l), fdiv_ru(a.u, b.u)};
        return {fdiv_rd(a.l, b.l), fdiv_ru(a.u, b.l)};
    }
    if (b.u < 0.f) {
        if (a.l >= 0.f) return {fdiv_rd(a.u, b.u), fdiv_ru(a.l, b.l)};
        if (a.u <= 0.f) return {fdiv_rd(a.u, b.l), fdiv_ru(a.l, b.u)};
        return {fdiv_rd(a.u, b.u), fdiv_ru(a.l, b.u)};
    }
    ok = false;
    return {-INFINITY, INFINITY};
}
// max / min of enclosed values (FP64 "x < y ? y : x" and "y < x ? y : x")
__device__ __forceinline__ E emax(E a, E b) { return {fmaxf(a.l, b.l), fmaxf(a.u, b.u)}; }
__device__ __forceinline__ E emin(E a, E b) { return {fminf(a.l, b.l), fminf(a.u, b.u)}; }

// certified FP64 comparisons of enclosed values
__device__ __forceinline__ bool clt(E a, E b, bool& ok) {
    if (a.u < b.l) return true;
    if (a.l >= b.u) return false;
    ok = false;
    return false;
}
__device__ __forceinline__ bool cle(E a, E b, bool& ok) {
    if (a.u <= b.l) return true;
    if (a.l > b.u) return false;
    ok = false;
    return false;
}

// n representable single steps toward -inf / +inf (finite y)
__device__ __forceinline__ float fstep_down(float y, int n) {
    int b = __float_as_int(y);
    if (y > 0.f) return b >= n ? __int_as_float(b - n) : __int_as_float((int)0x80000000u | (n - b));
    if (y < 0.f) return __int_as_float(b + n);
    return __int_as_float((int)0x80000000u | n);
}
__device__ __forceinline__ float fstep_up(float y, int n) { return -fstep_down(-y, n); }

// asinf padded kAsinfSteps single steps down / up: one shared (not inlined)
// copy each, like the FP64 asin, for the instruction caches
static __device__ __noinline__ float asinf_down(float x) { return fstep_down(asinf(x), kAsinfSteps); }
static __device__ __noinline__ float asinf_up(float x) { return fstep_up(asinf(x), kAsinfSteps); }

// enclosure of asin_rd64(v) and asin_ru64(v) for every FP64 v in x
__device__ __forceinline__ E easin(E x, bool& ok) {
    if (!(x.l >= -1.f && x.u <= 1.f)) {
        ok = false;
        return {-2.f, 2.f};
    }
    const float pi2 = 1.57079637f;  // >= 1.5707963267948968 (interval.cuh:366)
    float lo = asinf_down(x.l);
    float hi = asinf_up(x.u);
    if (lo < -pi2) lo = -pi2;
    if (x.l >= 0.f && lo < 0.f) lo = 0.f;
    if (hi > pi2) hi = pi2;
    if (x.u <= 0.f && hi > 0.f) hi = 0.f;
    return {lo, hi};
}

// an FP64 interval [lo, hi] with both bounds enclosed
struct EI {
    E lo, hi;
};
__device__ __forceinline__ EI ei(double lo, double hi) { return {ec(lo), ec(hi)}; }
__device__ __forceinline__ EI ept(E x) { return {x, x}; }
__device__ __forceinline__ EI iadd(EI a, EI b) { return {eadd(a.lo, b.lo), eadd(a.hi, b.hi)}; }
__device__ __forceinline__ EI isub(EI a, EI b) { return {esub(a.lo, b.hi), esub(a.hi, b.lo)}; }
// scaling by a positive constant is monotone: round the lower ends down and the
// upper ends up (exact for the powers of two used here, except near underflow)
__device__ __forceinline__ EI iscale(float n, EI a) {
    return {{__fmul_rd(a.lo.l, n), __fmul_ru(a.lo.u, n)}, {__fmul_rd(a.hi.l, n), __fmul_ru(a.hi.u, n)}};
}
// Three-valued comparison outcome of enclosed FP64 values.  Branches that only
// select between two values take the hull of both candidates when undecided.
enum Tri { T_FALSE = 0, T_TRUE = 1, T_UNKNOWN = 2 };
__device__ __forceinline__ int tlt(E a, E b) { return a.u < b.l ? T_TRUE : (a.l >= b.u ? T_FALSE : T_UNKNOWN); }
__device__ __forceinline__ int tle(E a, E b) { return a.u <= b.l ? T_TRUE : (a.l > b.u ? T_FALSE : T_UNKNOWN); }
__device__ __forceinline__ int tor(int x, int y) {
    return (x == T_TRUE || y == T_TRUE) ? T_TRUE : (x == T_FALSE && y == T_FALSE) ? T_FALSE : T_UNKNOWN;
}
__device__ __forceinline__ int tnot(int x) { return x == T_UNKNOWN ? x : 1 - x; }
__device__ __forceinline__ E hull(E a, E b) { return {fminf(a.l, b.l), fmaxf(a.u, b.u)}; }

// interval.hpp:214-231 + interval.cuh:352-355
__device__ __forceinline__ EI isq(EI x, bool& ok) {
    // l, u of the absolute value: each FP64 branch selects values only
    const int hpos = tlt(ek(0.f), x.hi), lneg = tlt(x.lo, ek(0.f));
    if (hpos == T_UNKNOWN || lneg == T_UNKNOWN) {
        // |x| bounds lie in the hull of all candidates: 0, |x.lo|, |x.hi|
        const E ax_lo = emax(x.lo, eneg(x.lo)), ax_hi = emax(x.hi, eneg(x.hi));
        const E u = emax(ax_lo, ax_hi);
        const E l = hull(ek(0.f), hull(ax_lo, ax_hi));
        return {emul(l, l), emul(u, u)};
    }
    E l = ek(0.f), u = ek(0.f);
    if (hpos == T_TRUE)
        u = x.hi;
    else
        l = eneg(x.hi);
    if (lneg == T_TRUE)
        u = emax(u, eneg(x.lo));
    else
        l = x.lo;
    return {emul(l, l), emul(u, u)};
}
// idiv_lo / idiv_hi (cp_fp64.cuh): the divisor's sign picks the case (a
// divisor possibly changing sign is handed to FP64); the dividend's sign only
// picks which quotient, so an undecided sign yields the hull of both.
__device__ __forceinline__ E pick_div(int t, E a1, E b1, E a2, E b2, bool& ok) {
    if (t == T_TRUE) return ediv(a1, b1, ok);
    if (t == T_FALSE) return ediv(a2, b2, ok);
    return hull(ediv(a1, b1, ok), ediv(a2, b2, ok));
}
__device__ __forceinline__ E idiv_lo(EI a, EI o, bool& ok) {
    const int pos = tlt(ek(0.f), o.lo), neg = tlt(o.hi, ek(0.f));
    if (pos == T_TRUE) return pick_div(tle(ek(0.f), a.lo), a.lo, o.hi, a.lo, o.lo, ok);
    if (pos == T_FALSE && neg == T_TRUE)
        return pick_div(tor(tle(ek(0.f), a.lo), tnot(tle(a.hi, ek(0.f)))), a.hi, o.hi, a.hi, o.lo, ok);
    if (pos == T_FALSE && neg == T_FALSE) return ek(-INFINITY);
    ok = false;
    return ek(-INFINITY);
}
__device__ __forceinline__ E idiv_hi(EI a, EI o, bool& ok) {
    const int pos = tlt(ek(0.f), o.lo), neg = tlt(o.hi, ek(0.f));
    if (pos == T_TRUE)
        return pick_div(tor(tle(ek(0.f), a.lo), tnot(tle(a.hi, ek(0.f)))), a.hi, o.lo, a.hi, o.hi, ok);
    if (pos == T_FALSE && neg == T_TRUE) return pick_div(tle(ek(0.f), a.lo), a.lo, o.lo, a.lo, o.hi, ok);
    if (pos == T_FALSE && neg == T_FALSE) return ek(INFINITY);
    ok = false;
    return ek(INFINITY);
}
__device__ __forceinline__ EI idiv(EI a, EI o, bool& ok) { return {idiv_lo(a, o, ok), idiv_hi(a, o, ok)}; }
__device__ __forceinline__ bool iempty(EI a, bool& ok) { return clt(a.hi, a.lo, ok); }
// tighten_lb / tighten_ub with an enclosed bound: the FP64 result is max / min
// of the two values whichever way the comparison goes, so no certification
__device__ __forceinline__ void tight_lo(EI& a, E x, bool&) { a.lo = emax(a.lo, x); }
__device__ __forceinline__ void tight_hi(EI& a, E x, bool&) { a.hi = emin(a.hi, x); }

// shadow of collision<W> (cp_fp64.cuh); trap events clear ok
__device__ __forceinline__ E collision_body(EI L, EI S, EI ab, const int W, bool& ok) {
    const bool HI = (W == W_HI);
    L.lo = emax(L.lo, S.lo);
    S.hi = emin(S.hi, L.hi);
    const EI l2 = isq(L, ok), s2 = isq(S, ok), a2 = isq(ab, ok);
    const EI sum = iadd(s2, a2);
    const bool obt_def = clt(sum.hi, l2.lo, ok);
    const bool obt_pos = clt(sum.lo, l2.hi, ok);
    EI add = idiv(isub(l2, s2), ab, ok);
    tight_lo(add, ek(0.f), ok);
    // Interval operations on proper intervals (lo <= hi) give proper intervals,
    // so the emptiness tests below reduce to comparisons of distinct quantities.
    // The callers pass proper L, S with S.lo <= L.hi (so both stay proper after
    // the two tightenings above); with S.lo > 0 and ab.lo > 0, add.hi =
    // ru(ru(L.hi^2) - rd(S.lo^2)) / ab >= 0, so add stays proper after its own.
    if (!(clt(ek(0.f), S.lo, ok) && clt(ek(0.f), ab.lo, ok))) ok = false;
    if (!ok) return ek(0.f);

    bool ob_set = false;
    E ob_val = ek(HI ? -1.f : 0.f);
    EI lq{ek(0.f), ek(0.f)}, sq{ek(0.f), ek(0.f)};
    if (obt_pos) {
        EI lx = iscale(0.5f, iadd(add, ab));
        EI sx = iscale(0.5f, isub(add, ab));
        // [max(lo, 0), min(hi, S.hi)] of a proper interval is empty iff
        // hi < 0, lo > S.hi or S.hi < 0; [lo, min(hi, L.hi)] iff lo > L.hi
        const bool e1 = clt(sx.hi, ek(0.f), ok) || clt(S.hi, sx.lo, ok) || clt(S.hi, ek(0.f), ok);
        const bool e2 = e1 ? false : clt(L.hi, lx.lo, ok);
        tight_lo(sx, ek(0.f), ok);
        tight_hi(sx, S.hi, ok);
        tight_hi(lx, L.hi, ok);
        if (e1 || e2) {
            if (obt_def) ok = false;  // trap site
        } else {
            lq = idiv(lx, L, ok);
            sq = idiv(sx, S, ok);
            // quotients of proper, non-empty intervals are proper: [lo, min(hi, 1)]
            // is empty iff lo > 1
            const bool e3 = clt(ek(1.f), lq.lo, ok);
            const bool e4 = e3 ? false : clt(ek(1.f), sq.lo, ok);
            tight_hi(lq, ek(1.f), ok);
            tight_hi(sq, ek(1.f), ok);
            if (e3 || e4) {
                if (obt_def) ok = false;
            } else {
                if (clt(lq.lo, ek(-1.f), ok) || clt(ek(1.f), lq.hi, ok) || clt(sq.lo, ek(-1.f), ok) ||
                    clt(ek(1.f), sq.hi, ok))
                    ok = false;
                ob_set = true;
                if (W == W_TRAP) {
                } else if (HI) {
                    ob_val = esub(easin(lq.hi, ok), easin(sq.lo, ok));
                } else {
                    ob_val = emax(esub(easin(lq.lo, ok), easin(sq.hi, ok)), ek(0.f));
                }
            }
        }
    }
    if (!ok) return ek(0.f);
    if (!obt_def) {
        EI lx = iscale(0.5f, iadd(ab, add));
        EI sx = iscale(0.5f, isub(ab, add));
        const bool e5 = clt(sx.hi, ek(0.f), ok);  // [max(lo, 0), hi] empty iff hi < 0
        tight_lo(sx, ek(0.f), ok);
        if (e5) {
            if (!obt_pos) ok = false;
        } else {
            if (W == W_TRAP) {
                EI alq = idiv(lx, L, ok), asq = idiv(sx, S, ok);
                if (clt(alq.lo, ek(-1.f), ok) || clt(ek(1.f), alq.hi, ok) || clt(asq.lo, ek(-1.f), ok) ||
                    clt(ek(1.f), asq.hi, ok))
                    ok = false;
                return ek(0.f);
            }
            E r;
            if (HI) {
                const E lqh = idiv_hi(lx, L, ok), sqh = idiv_hi(sx, S, ok);
                if (clt(ek(1.f), lqh, ok) || clt(ek(1.f), sqh, ok)) ok = false;
                const bool lx_nonneg = cle(ek(0.f), lx.lo, ok) && clt(ek(0.f), L.lo, ok);
                if (!lx_nonneg && clt(idiv_lo(lx, L, ok), ek(-1.f), ok)) ok = false;
                const bool sx_nonneg = cle(ek(0.f), sx.lo, ok) && clt(ek(0.f), S.lo, ok);
                if (!sx_nonneg && clt(idiv_lo(sx, S, ok), ek(-1.f), ok)) ok = false;
                r = eadd(easin(lqh, ok), easin(sqh, ok));
            } else {
                const EI alq = idiv(lx, L, ok), asq = idiv(sx, S, ok);
                if (clt(alq.lo, ek(-1.f), ok) || clt(ek(1.f), alq.hi, ok) || clt(asq.lo, ek(-1.f), ok) ||
                    clt(ek(1.f), asq.hi, ok))
                    ok = false;
                r = eadd(easin(alq.lo, ok), emax(easin(asq.lo, ok), ek(0.f)));
            }
            // result.empty() ? r : join(result, r): both candidates are values, so an
            // undecided emptiness takes their hull
            int nonempty;
            if (!ob_set) {
                nonempty = T_FALSE;
            } else if (HI) {
                nonempty = tnot(tlt(ob_val, ek(0.f)));
            } else {
                nonempty = tle(sq.lo, lq.hi);
                if (nonempty != T_TRUE)
                    nonempty = tor(nonempty, tnot(tlt(esub(easin(lq.hi, ok), easin(sq.lo, ok)), ek(0.f))));
            }
            const E joined = HI ? emax(ob_val, r) : emin(ob_val, r);
            ob_val = nonempty == T_TRUE ? joined : nonempty == T_FALSE ? r : hull(joined, r);
        }
    }
    return ob_val;
}

// One shared (not inlined) copy per Want, with the certification flag in a
// register of its own: a flag passed by reference into an out-of-line function
// lives in local memory, and the shadow reads it after almost every step.
struct EOk {
    E v;
    bool ok;
};
// one copy for all three Wants (a runtime argument), for the instruction caches
static __device__ __noinline__ EOk collision_call(EI L, EI S, EI ab, int W) {
    bool ok = true;
    const E v = collision_body(L, S, ab, W, ok);
    return {v, ok};
}
template <int W>
__device__ __forceinline__ E collision(EI L, EI S, EI ab, bool& ok) {
    const EOk r = collision_call(L, S, ab, W);
    ok = ok && r.ok;
    return r.v;
}

// corner wrappers (shadows of cp_fp64.cuh); LOC = lower-bound corner, which
// returns 0 when the radii sum is not positive (collision_angles.cu:131-137, 222-228)
// ra, rb: the exact FP64 corner radii; ra >= rb makes the corner intervals
// (one directed sum each) satisfy shorter.lo <= longer.hi
template <int W, bool LOC>
__device__ __forceinline__ E ca_ii_corner(double la, double ra, double rb, bool& ok) {
    const E eR = ec(ra), eS = ec(rb), eL = ec(la);
    EI lc = ept(eadd(eR, eL)), sc = ept(eadd(eS, eL)), ab = ept(eadd(eR, eS));
    if (LOC && cle(ab.lo, ek(0.f), ok)) return ek(0.f);
    if (!(ra >= rb)) ok = false;
    return collision<W>(lc, sc, ab, ok);
}
template <int W, bool LOC>
__device__ __forceinline__ E ca_oo_corner(double ra, double rb, bool& ok) {
    const E eR = ec(ra), eS = ec(rb);
    EI lc = ept(esub(ek(1.f), eS)), sc = ept(esub(ek(1.f), eR)), ab = ept(eadd(eR, eS));
    if (LOC && cle(ab.lo, ek(0.f), ok)) return ek(0.f);
    if (!(ra >= rb)) ok = false;
    return collision<W>(lc, sc, ab, ok);
}
template <int W, bool OUTER_FIRST>
__device__ __forceinline__ E ca_mixed_corner(EI la, E a, E b, bool& ok) {
    EI ca, cb;
    if (OUTER_FIRST) {
        ca = ept(esub(ek(1.f), a));
        cb = {eadd(la.lo, b), eadd(la.hi, b)};
    } else {
        ca = {eadd(la.lo, a), eadd(la.hi, a)};
        cb = ept(esub(ek(1.f), b));
    }
    EI ab = ept(eadd(a, b));
    const bool def_ca_longer = cle(cb.hi, ca.lo, ok);
    const bool pos_ca_longer = cle(cb.lo, ca.hi, ok);
    if (def_ca_longer) return collision<W>(ca, cb, ab, ok);
    if (!pos_ca_longer) return collision<W>(cb, ca, ab, ok);
    const E r1 = collision<W>(ca, cb, ab, ok);
    const E r2 = collision<W>(cb, ca, ab, ok);
    return (W == W_HI) ? emax(r1, r2) : emin(r1, r2);
}
template <bool OUTER_FIRST, int W = W_LO>
__device__ __forceinline__ E ca_mixed_lo(EI la, EI ra, EI rb, bool& ok) {
    const E lhs = emul(eadd(ra.lo, rb.lo), ek(2.f));
    const E rhs = esub(ek(1.f), la.lo);
    if (cle(lhs, rhs, ok)) return ek(0.f);
    return ca_mixed_corner<W, OUTER_FIRST>(la, ra.lo, rb.lo, ok);
}
template <bool OUTER_FIRST, int W = W_HI>
__device__ __forceinline__ E ca_mixed_hi(EI la, EI ra, EI rb, bool& ok) {
    return ca_mixed_corner<W, OUTER_FIRST>(la, ra.hi, rb.hi, ok);
}
// a box axis: exact FP64 bounds and their enclosures
struct BI {
    double lo, hi;
    EI e;
};
__device__ __forceinline__ BI bi(double lo, double hi) { return {lo, hi, ei(lo, hi)}; }
__device__ __forceinline__ EI ca_inner_inner(const BI& la, const BI& ra, const BI& rb, bool& ok) {
    const E hi = ca_ii_corner<W_HI, false>(la.lo, ra.hi, rb.hi, ok);
    return {ca_ii_corner<W_LO, true>(la.hi, ra.lo, rb.lo, ok), hi};
}
__device__ __forceinline__ EI ca_outer_outer(const BI& ra, const BI& rb, bool& ok) {
    const E hi = ca_oo_corner<W_HI, false>(ra.hi, rb.hi, ok);
    return {ca_oo_corner<W_LO, true>(ra.lo, rb.lo, ok), hi};
}
__device__ __forceinline__ EI ca_outer_inner(EI la, EI ra, EI rb, bool& ok) {
    return {ca_mixed_lo<true>(la, ra, rb, ok), ca_mixed_hi<true>(la, ra, rb, ok)};
}
__device__ __forceinline__ EI ca_inner_outer(EI la, EI ra, EI rb, bool& ok) {
    return {ca_mixed_lo<false>(la, ra, rb, ok), ca_mixed_hi<false>(la, ra, rb, ok)};
}
__device__ __forceinline__ E semi_outer_lo(EI r, bool& ok) {
    return easin(ediv(r.lo, esub(ek(1.f), r.lo), ok), ok);
}
__device__ __forceinline__ E semi_outer_hi(EI r, bool& ok) {
    return easin(ediv(r.hi, esub(ek(1.f), r.hi), ok), ok);
}
__device__ __forceinline__ E semi_inner_lo(EI la, EI r, bool& ok) {
    return easin(ediv(r.lo, eadd(la.hi, r.lo), ok), ok);
}
__device__ __forceinline__ E semi_inner_hi(EI la, EI r, bool& ok) {
    return easin(ediv(r.hi, eadd(la.lo, r.hi), ok), ok);
}
__device__ __forceinline__ E kcr() { return {0.564199984f, 0.564200044f}; }  // encloses 0.5642
__device__ __forceinline__ E klbpi() { return {3.14159250f, 3.14159274f}; }  // encloses 3.141592653589793
__device__ __forceinline__ E area_ratio_ub(EI la) { return esub(ek(1.f), emul(la.lo, la.lo)); }
__device__ __forceinline__ E disk_area_lb(EI r) { return emul(klbpi(), emul(r.lo, r.lo)); }
__device__ __forceinline__ E used_ub(E ratio, E angle_hi) { return emul(ratio, emul(ek(0.5f), angle_hi)); }
// FP64 "lhs >= rhs" and "lhs < rhs", certified
__device__ __forceinline__ bool holds(E lhs, E rhs, bool& ok) { return !clt(lhs, rhs, ok); }

// ---------------------------------------------------------------- families
// handle_case_1_1 / handle_case_2_1 (middle_configuration.cu:86-154); true = failed
__device__ __forceinline__ bool middle_handle_body(const BI& Bla, const BI& Br1, const BI& Br2, const BI& Br3, bool inner_first,
                                             bool& ok, int* sub) {
    const EI la = Bla.e, r1 = Br1.e, r2 = Br2.e, r3 = Br3.e;
    const E ratio = area_ratio_ub(la);
    const E a1 = disk_area_lb(r1), a2 = disk_area_lb(r2);
    E c12_hi, c23_hi, c13_lo;
    if (inner_first) {
        c12_hi = ca_mixed_hi<false>(la, r1, r2, ok);
        c13_lo = ca_ii_corner<W_LO, true>(Bla.hi, Br1.lo, Br3.lo, ok);
        c23_hi = ca_mixed_hi<true>(la, r2, r3, ok);
    } else {
        c12_hi = ca_mixed_hi<true>(la, r1, r2, ok);
        c13_lo = ca_oo_corner<W_LO, true>(Br1.lo, Br3.lo, ok);
        c23_hi = ca_mixed_hi<false>(la, r2, r3, ok);
    }
    if (!ok) return false;
    if (cle(c13_lo, eadd(c12_hi, c23_hi), ok)) {
        const E lhs = emul(ek(0.5f), eadd(a1, a2));
        const E rhs = emul(kcr(), used_ub(ratio, c12_hi));
        if (clt(lhs, rhs, ok)) {
            *sub = 0;
            return true;
        }
    }
    if (!ok) return false;
    E c12_lo, c23_lo, c13_hi;
    if (inner_first) {
        c12_lo = ca_mixed_lo<false>(la, r1, r2, ok);
        c13_hi = ca_ii_corner<W_HI, false>(Bla.lo, Br1.hi, Br3.hi, ok);
        c23_lo = ca_mixed_lo<true>(la, r2, r3, ok);
    } else {
        c12_lo = ca_mixed_lo<true>(la, r1, r2, ok);
        c13_hi = ca_oo_corner<W_HI, false>(Br1.hi, Br3.hi, ok);
        c23_lo = ca_mixed_lo<false>(la, r2, r3, ok);
    }
    if (!cle(c13_hi, eadd(c12_lo, c23_lo), ok)) {
        const E a3 = disk_area_lb(r3);
        const E lhs = eadd(emul(ek(0.5f), eadd(a1, a3)), a2);
        const E rhs = emul(kcr(), used_ub(ratio, c13_hi));
        if (clt(lhs, rhs, ok)) {
            *sub = 1;
            return true;
        }
    }
    return false;
}

template <bool INNER>
__device__ __forceinline__ bool end2d_handle_body(EI la, EI r1, EI r2, bool& ok) {
    EI ca, sa;
    E other_hi, rho_lo;
    if (INNER) {
        ca = ca_inner_outer(la, r1, r2, ok);
        sa = {semi_outer_lo(r2, ok), semi_outer_hi(r2, ok)};
        other_hi = semi_inner_hi(la, r1, ok);
        const EI t = isub(ept(ek(1.f)), iscale(2.f, r2));
        rho_lo = esub(isq(t, ok).lo, isq(la, ok).hi);
    } else {
        ca = ca_outer_inner(la, r1, r2, ok);
        sa = {semi_inner_lo(la, r2, ok), semi_inner_hi(la, r2, ok)};
        other_hi = semi_outer_hi(r1, ok);
        rho_lo = esub(ek(1.f), isq(iadd(la, iscale(2.f, r2)), ok).hi);
    }
    const EI a = iadd(ca, sa);
    const E used = used_ub(area_ratio_ub(la), a.hi);
    rho_lo = emax(rho_lo, ek(0.f));
    const E alpha = esub(a.lo, other_hi);
    const E reusable = emul(emul(ek(0.5f), alpha), rho_lo);
    const E lhs = eadd(disk_area_lb(r2), emul(ek(0.5f), disk_area_lb(r1)));
    const E rhs = emul(kcr(), esub(used, reusable));
    return !holds(lhs, rhs, ok);
}

template <bool INNER>
__device__ __forceinline__ bool end3d_handle_body(const BI& Bla, const BI& Br1, const BI& Br2, const BI& Br3, bool& ok) {
    const EI la = Bla.e, r1 = Br1.e, r2 = Br2.e, r3 = Br3.e;
    E a12_lo, a23_lo, a13_hi;
    if (INNER) {
        a12_lo = ca_mixed_lo<false>(la, r1, r2, ok);
        a23_lo = ca_mixed_lo<true>(la, r2, r3, ok);
        a13_hi = ca_ii_corner<W_HI, false>(Bla.lo, Br1.hi, Br3.hi, ok);
        ca_mixed_hi<true, W_TRAP>(la, r2, r3, ok);
    } else {
        a12_lo = ca_mixed_lo<true>(la, r1, r2, ok);
        a23_lo = ca_mixed_lo<false>(la, r2, r3, ok);
        a13_hi = ca_oo_corner<W_HI, false>(Br1.hi, Br3.hi, ok);
        ca_mixed_hi<false, W_TRAP>(la, r2, r3, ok);
    }
    if (!ok) return false;
    if (cle(a13_hi, eadd(a12_lo, a23_lo), ok)) {
        if (INNER) {
            ca_mixed_hi<false, W_TRAP>(la, r1, r2, ok);
            ca_ii_corner<W_TRAP, true>(Bla.hi, Br1.lo, Br3.lo, ok);
        } else {
            ca_mixed_hi<true, W_TRAP>(la, r1, r2, ok);
            ca_oo_corner<W_TRAP, true>(Br1.lo, Br3.lo, ok);
        }
        return false;
    }
    E a12_hi, a13_lo, a2_hi, rho_lo;
    EI a3;
    if (INNER) {
        a12_hi = ca_mixed_hi<false>(la, r1, r2, ok);
        a13_lo = ca_ii_corner<W_LO, true>(Bla.hi, Br1.lo, Br3.lo, ok);
        a3 = {semi_inner_lo(la, r3, ok), semi_inner_hi(la, r3, ok)};
        a2_hi = semi_outer_hi(r2, ok);
        rho_lo = esub(ek(1.f), isq(iadd(la, iscale(2.f, r3)), ok).hi);
    } else {
        a12_hi = ca_mixed_hi<true>(la, r1, r2, ok);
        a13_lo = ca_oo_corner<W_LO, true>(Br1.lo, Br3.lo, ok);
        a3 = {semi_outer_lo(r3, ok), semi_outer_hi(r3, ok)};
        a2_hi = semi_inner_hi(la, r2, ok);
        const EI t = isub(ept(ek(1.f)), iscale(2.f, r3));
        rho_lo = esub(isq(t, ok).lo, isq(la, ok).hi);
    }
    const EI a = iadd(EI{a13_lo, a13_hi}, a3);
    const E reusable_alpha_lo = esub(a.lo, eadd(a12_hi, a2_hi));
    rho_lo = emax(rho_lo, ek(0.f));
    const E reusable = emul(emul(ek(0.5f), reusable_alpha_lo), rho_lo);
    const E used = used_ub(area_ratio_ub(la), a.hi);
    const E lhs = eadd(eadd(disk_area_lb(r2), disk_area_lb(r3)), emul(ek(0.5f), disk_area_lb(r1)));
    const E rhs = emul(kcr(), esub(used, reusable));
    return !holds(lhs, rhs, ok);
}

// Out-of-line handles (one copy each) taking their boxes by value and returning
// a packed status, so no flag or box lives in local memory: -2 = not certified,
// -1 = the handle holds, k >= 0 = sub-check k fails.
static __device__ __noinline__ int middle_handle_call(BI Bla, BI Br1, BI Br2, BI Br3, bool inner_first) {
    bool ok = true;
    int sub = 0;
    const bool failed = middle_handle_body(Bla, Br1, Br2, Br3, inner_first, ok, &sub);
    return !ok ? -2 : failed ? sub : -1;
}
template <bool INNER>
__device__ __noinline__ int end2d_handle_call(EI la, EI r1, EI r2) {
    bool ok = true;
    const bool failed = end2d_handle_body<INNER>(la, r1, r2, ok);
    return !ok ? -2 : failed ? 0 : -1;
}
template <bool INNER>
__device__ __noinline__ int end3d_handle_call(BI Bla, BI Br1, BI Br2, BI Br3) {
    bool ok = true;
    const bool failed = end3d_handle_body<INNER>(Bla, Br1, Br2, Br3, ok);
    return !ok ? -2 : failed ? 0 : -1;
}

}  // namespace f32

// The FP32 shadow of eval_box<FAM, DECIDE> (cp_families.cuh).  Returns the
// FP64 DECIDE verdict (and its mask in *mask) when it is certain, PF_UNDECIDED
// otherwise.  With proved_only, only PROVED / EMPTY are issued (FULL-mode
// callers need the complete FP64 mask of every other box).
template <int FAM>
__device__ __forceinline__ int prefilter_box(const double* lo, const double* hi, int order, bool proved_only,
                                             uint8_t* mask) {
    using namespace f32;
    constexpr int D = family_dims(FAM);
    *mask = 0;
    // tightening, emptiness and the fit check stay in FP64: they are exact and cheap
    double l1 = lo[1], l2 = lo[2];
    if (D == 4 && l2 < lo[3]) l2 = lo[3];
    if (l1 < l2) l1 = l2;
    if (lo[0] > hi[0] || l1 > hi[1] || l2 > hi[2] || (D == 4 && lo[3] > hi[3])) return PF_EMPTY;
    const bool has_fit = FAM != F_START_END_2D && FAM != F_START_END_3D;
    const bool fit_fires = has_fit && __dmul_ru(2.0, hi[1]) >= __dadd_rd(1.0, -hi[0]);
    if (fit_fires) {
        if (FAM != F_START) {
            if (proved_only) return PF_UNDECIDED;
            *mask = M_FIT;
            return PF_NOFIT;
        }
    }
    const uint8_t fit_bit = fit_fires ? M_FIT : 0;
    const BI Bla = bi(lo[0], hi[0]), Br1 = bi(l1, hi[1]), Br2 = bi(l2, hi[2]);
    const BI Br3 = D == 4 ? bi(lo[3], hi[3]) : bi(0.0, 0.0);
    const EI la = Bla.e, r1 = Br1.e, r2 = Br2.e, r3 = Br3.e;
    bool ok = true;
    int fail_bit = -1;
    if (FAM == F_START) {
        const EI a12 = ca_outer_inner(la, r1, r2, ok);
        const EI a13 = ca_outer_outer(Br1, Br3, ok);
        const EI a23 = ca_inner_outer(la, r2, r3, ok);
        const EI s = iadd(a12, a23);
        const bool c_def = clt(a13.hi, s.lo, ok), c_pos = clt(a13.lo, s.hi, ok);
        const E ratio = area_ratio_ub(la);
        const E ar1 = disk_area_lb(r1), ar2 = disk_area_lb(r2);
        const E so_hi = semi_outer_hi(r1, ok);
        if (c_pos && ok) {
            const E lhs = eadd(ar1, emul(ek(0.5f), ar2));
            const E rhs = emul(kcr(), used_ub(ratio, eadd(so_hi, a12.hi)));
            if (!holds(lhs, rhs, ok)) fail_bit = 0;
        }
        if (fail_bit < 0 && !c_def && ok) {
            const E lhs = eadd(eadd(ar1, ar2), emul(ek(0.5f), disk_area_lb(r3)));
            const E rhs = emul(kcr(), used_ub(ratio, eadd(so_hi, a13.hi)));
            if (!holds(lhs, rhs, ok)) fail_bit = 1;
        }
    } else if (FAM == F_START_END_2D) {
        const E a1_hi = semi_outer_hi(r1, ok);
        const EI a2{semi_inner_lo(la, r2, ok), semi_inner_hi(la, r2, ok)};
        const EI a12 = ca_outer_inner(la, r1, r2, ok);
        const E total_hi = eadd(eadd(a1_hi, a2.hi), a12.hi);
        const E reuse_lo = emax(esub(eadd(a12.lo, a2.lo), a1_hi), ek(0.f));
        const E used = used_ub(area_ratio_ub(la), total_hi);
        const E rho_lo = emax(esub(ek(1.f), isq(iadd(la, iscale(2.f, r2)), ok).hi), ek(0.f));
        const E reusable = emul(emul(ek(0.5f), reuse_lo), rho_lo);
        const E lhs = eadd(disk_area_lb(r2), disk_area_lb(r1));
        const E rhs = emul(kcr(), esub(used, reusable));
        if (!holds(lhs, rhs, ok)) fail_bit = 0;
    } else if (FAM == F_START_END_3D) {
        const EI a1{semi_outer_lo(r1, ok), semi_outer_hi(r1, ok)};
        const EI a2{semi_inner_lo(la, r2, ok), semi_inner_hi(la, r2, ok)};
        const EI a3{semi_outer_lo(r3, ok), semi_outer_hi(r3, ok)};
        const EI a12 = ca_outer_inner(la, r1, r2, ok);
        const EI a13 = ca_outer_outer(Br1, Br2, ok);
        const EI a23 = ca_inner_outer(la, r2, r3, ok);
        const EI b123 = iadd(a12, a23);
        const EI b13{emax(a13.lo, b123.lo), emax(a13.hi, b123.hi)};
        const EI a123 = iadd(iadd(a1, b13), a3);
        const EI a122 = iadd(iadd(a1, a12), a2);
        const EI a{emax(a123.lo, a122.lo), emax(a123.hi, a122.hi)};
        const E reuse_angle = emax(esub(a.lo, a122.hi), ek(0.f));
        const E outer_rad = esub(ek(1.f), emul(ek(2.f), r3.hi));
        const E outer_sq = emul(outer_rad, outer_rad);
        const E inner_sq = emul(la.hi, la.hi);
        const E reused = emax(emul(emul(ek(0.5f), reuse_angle), esub(outer_sq, inner_sq)), ek(0.f));
        const E used = esub(used_ub(area_ratio_ub(la), a.hi), reused);
        const E lhs = eadd(disk_area_lb(r1), eadd(disk_area_lb(r2), disk_area_lb(r3)));
        const E rhs = emul(kcr(), used);
        if (!holds(lhs, rhs, ok)) fail_bit = 0;
    } else if (FAM == F_MIDDLE) {
        const bool second_first = (order & 1) != 0;
        for (int h = 0; h < 2 && ok && fail_bit < 0; ++h) {
            const bool inner = (h == 0) != second_first;
            const int r = middle_handle_call(Bla, Br1, Br2, Br3, inner);
            if (r == -2)
                ok = false;
            else if (r >= 0)
                fail_bit = (inner ? 0 : 2) + r;
        }
    } else if (FAM == F_END_2D) {
        const bool second_first = (order & 1) != 0;
        for (int h = 0; h < 2 && ok && fail_bit < 0; ++h) {
            const bool inner = (h == 0) != second_first;
            const int r = inner ? end2d_handle_call<true>(la, r1, r2) : end2d_handle_call<false>(la, r1, r2);
            if (r == -2)
                ok = false;
            else if (r >= 0)
                fail_bit = inner ? 0 : 1;
        }
    } else if (FAM == F_END_3D) {
        const bool second_first = (order & 1) != 0;
        for (int h = 0; h < 2 && ok && fail_bit < 0; ++h) {
            const bool inner = (h == 0) != second_first;
            const int r = inner ? end3d_handle_call<true>(Bla, Br1, Br2, Br3) : end3d_handle_call<false>(Bla, Br1, Br2, Br3);
            if (r == -2)
                ok = false;
            else if (r >= 0)
                fail_bit = inner ? 0 : 1;
        }
    }
    if (!ok) return PF_UNDECIDED;
    if (fail_bit >= 0) {
        if (proved_only) return PF_UNDECIDED;
        *mask = (uint8_t)(fit_bit | (1u << fail_bit));
        return PF_CRITICAL;
    }
    *mask = fit_bit;
    return PF_PROVED;
}

}  // namespace cpb
