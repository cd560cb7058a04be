// Device-resident worklist pieces: box storage, child generation (bisection
// clipped to the family's dependent ranges) and warp-aggregated appends.
#pragma once
#include "cp_families.cuh"
#include "cp_lattice.cuh"

namespace cpb {

// Structure-of-arrays box list: axis d of box i is lo[d*cap + i] / hi[d*cap + i].
// aux (optional, start family): the lambda-independent criterion terms of box
// i, LaFree field k at aux[k*cap + i] (a13.lo, a13.hi, semi-angle of r1, flag),
// carried from a box to those of its children whose radii are unchanged.
struct BoxList {
    double* lo;
    double* hi;
    uint8_t* depth;
    size_t cap;
    double* aux = nullptr;  // a list built member by member carries no terms
};
constexpr int kAuxFields = 4;

// Split policies (how a not-proved box is refined)
enum SplitPolicy : int {
    SPLIT_UNIFORM = 0,  // bisect every axis: 2^dims children
    SPLIT_LAMBDA = 1,   // bisect lambda only (the reference refines lambda only, run_kernel.cuh:110-127)
    SPLIT_WIDEST = 2,   // bisect the axis with the largest width relative to its scale
    SPLIT_GIVEN = 3,    // bisect the axis chosen per box by the learned model
    SPLIT_HYBRID = 4    // lambda while wider than its target width, else the widest radius
};

// Single-placement bounds on a uniform lambda grid t_i = 0.5 + i*h, i = 0..n-1,
// used to clip child boxes: the bound is non-increasing in lambda, so the value
// at the largest grid point t_i <= lambda.lo is an upper bound for the box.
struct SingleTable {
    const double* t;  // grid points
    const double* v;  // single_placement(t_i)
    int n;
    double h;
};

__device__ __forceinline__ double single_upper(const SingleTable& tab, double la_lo) {
    if (!(la_lo >= tab.t[0])) return 0.25;  // the bisection never exceeds 0.25
    int i = (int)((la_lo - tab.t[0]) / tab.h);
    if (i >= tab.n) i = tab.n - 1;
    while (i > 0 && tab.t[i] > la_lo) --i;
    while (i + 1 < tab.n && tab.t[i + 1] <= la_lo) ++i;
    return tab.v[i];
}

// Intersects a child box with the dependent ranges of its own lambda interval
// (the ranges the family lattice enumerates, e.g. middle_configuration.cu:66-84).
// Returns false when the child contains no configuration.
template <int FAM>
__device__ __forceinline__ bool clip_child(double* lo, double* hi, const SingleTable& tab) {
    constexpr int D = family_dims(FAM);
    const Iv la{lo[0], hi[0]};
    const Iv r1r = range_r1(la, single_upper(tab, la.lo));
    if (lo[1] < r1r.lo) lo[1] = r1r.lo;
    if (r1r.hi < hi[1]) hi[1] = r1r.hi;
    if (lo[1] > hi[1]) return false;
    const Iv r2r = range_r2(FAM, la, Iv{lo[1], hi[1]});
    if (lo[2] < r2r.lo) lo[2] = r2r.lo;
    if (r2r.hi < hi[2]) hi[2] = r2r.hi;
    if (lo[2] > hi[2]) return false;
    if (D == 4) {
        const Iv r3r = range_r3(FAM, la, Iv{lo[2], hi[2]});
        if (lo[3] < r3r.lo) lo[3] = r3r.lo;
        if (r3r.hi < hi[3]) hi[3] = r3r.hi;
        if (lo[3] > hi[3]) return false;
    }
    return true;
}

__device__ __forceinline__ double midpoint(double a, double b) { return __dmul_rn(0.5, __dadd_rn(a, b)); }

// Axis with the largest width relative to its scale: lambda against the lane
// width 1 - lambda, radii against their upper bound.
template <int D>
__device__ __forceinline__ int widest_axis(const double* lo, const double* hi) {
    double best = (hi[0] - lo[0]) / fmax(1.0 - hi[0], 1e-300);
    int ax = 0;
#pragma unroll
    for (int d = 1; d < D; ++d) {
        double w = (hi[d] - lo[d]) / fmax(hi[d], 1e-300);
        if (w > best) {
            best = w;
            ax = d;
        }
    }
    return ax;
}

// Hybrid rule: the width lambda needs shrinks about like (1 - lambda)^2 toward
// the top of the domain; above `scale * (1 - la.hi)^2` lambda is bisected,
// below it the radius whose width is largest relative to the lane width.
template <int D>
__device__ __forceinline__ int hybrid_axis(const double* lo, const double* hi, double scale) {
    const double lane = 1.0 - hi[0];
    if (hi[0] - lo[0] > scale * lane * lane) return 0;
    int ax = 1;
    double best = hi[1] - lo[1];
#pragma unroll
    for (int d = 2; d < D; ++d)
        if (hi[d] - lo[d] > best) {
            best = hi[d] - lo[d];
            ax = d;
        }
    return ax;
}

// Number of children a split produces before clipping.
__host__ __device__ constexpr int fanout(int policy, int dims) { return policy == SPLIT_UNIFORM ? (1 << dims) : 2; }

// Writes child c (0 <= c < fanout) of box (lo, hi) split on `axis` (binary
// policies) or on every axis (uniform).
template <int D>
__device__ __forceinline__ void make_child(const double* lo, const double* hi, int policy, int axis, int c, double* clo,
                                           double* chi) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
        clo[d] = lo[d];
        chi[d] = hi[d];
    }
    if (policy == SPLIT_UNIFORM) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double m = midpoint(lo[d], hi[d]);
            if ((c >> d) & 1)
                clo[d] = m;
            else
                chi[d] = m;
        }
    } else {
        const double m = midpoint(lo[axis], hi[axis]);
        if (c & 1)
            clo[axis] = m;
        else
            chi[axis] = m;
    }
}

// Warp-aggregated reservation of `count` slots; returns this lane's first slot
// (only meaningful for lanes with count > 0).  All lanes of the warp take part.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* counter, unsigned count) {
    const unsigned lane = threadIdx.x & 31;
    unsigned incl = count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= (unsigned)off) incl += v;
    }
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total) base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    return base + (incl - count);
}

// As warp_reserve, for writers that emit the warp's slots cooperatively:
// returns the warp's first slot; *excl = this lane's offset in the warp's range,
// *total = the warp's slot count (uniform).  All lanes of the warp take part.
__device__ __forceinline__ unsigned long long warp_reserve_range(unsigned long long* counter, unsigned count,
                                                                 unsigned* excl, unsigned* total) {
    const unsigned lane = threadIdx.x & 31;
    unsigned incl = count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= (unsigned)off) incl += v;
    }
    *total = __shfl_sync(0xffffffffu, incl, 31);
    *excl = incl - count;
    unsigned long long base = 0;
    if (lane == 31 && *total) base = atomicAdd(counter, (unsigned long long)*total);
    return __shfl_sync(0xffffffffu, base, 31);
}

}  // namespace cpb
