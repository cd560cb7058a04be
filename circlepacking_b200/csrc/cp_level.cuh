// The level step of the box refinement, shared by the level-synchronous
// kernel (cp_engine.cu) and the persistent graph-driven kernel (cp_graph.cu):
// evaluate one box per lane (DECIDE mode, optional FP32 pre-pass and per-box
// criterion order), count verdicts, and append the children of every box that
// is not proved to the next worklist level.
#pragma once
#include <cstdint>

#include "cp_prover.h"
#include "cp_fp32.cuh"
#include "cp_worklist.cuh"

namespace cpb {

// counter block layout (unsigned long long)
enum : int {
    C_VERDICT = 0,  // 5 verdict counts
    C_UNRESOLVED = 5,
    C_CLIPPED = 6,
    C_FP32 = 7,
    C_OUT = 8,      // children appended
    C_ERR = 9,      // error flags
    C_BEST_SLAB = 10,
    C_EVALUATED = 11,
    C_FIRST_BITS = 12,  // ordered encoding of the smallest failing lambda.lb
    C_ERRBOX_CLAIM = 13,
    C_ERRBOX = 14,      // 8 slots: lo/hi of the first erroneous box
    C_COLLECT = 22,
    C_NOFIT_SLAB = 23,  // smallest lambda slab holding a box whose fit check fired (middle/end)
    C_TRAP_SLAB = 24,   // smallest lambda slab holding a box that reached a trap site
    C_HANDLES = 25,     // guarded criteria evaluated in FP64
    C_DIGEST = 26,      // 2 words: sum and xor of the per-box verdict hashes (when enabled)
    C_COUNT = 28
};
enum : unsigned long long { E_OVERFLOW = 1, E_NOFIT = 2, E_TRAP = 4, E_TC = 8 /* tensor-core wait timed out */ };
constexpr int kDepthBins = 64;

struct LevelArgs {
    BoxList in;
    size_t begin, count;
    BoxList out;
    unsigned long long* cnt;
    unsigned long long* per_depth;
    SingleTable tab;
    int policy, max_depth;
    double lambda_scale;        // SPLIT_HYBRID
    const uint8_t* axis_hint;   // per input box (SPLIT_GIVEN), indexed from `begin`
    const uint8_t* order_hint;  // per input box criterion order, or null
    int digest;                 // 1: fold every evaluated (box, verdict) pair into the digest counters
};

// Order-independent digest of a set of (box, verdict) pairs: each evaluated box
// contributes a 64-bit hash of the bit patterns of its bounds and its verdict,
// summed (mod 2^64) and, after a second finalisation, xor-ed into two counters.
// Two refinements that evaluate the same boxes with the same verdicts give the
// same pair of words in any order.  The mixing step is the splitmix64 finaliser
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators", 2014).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
template <int D>
__device__ __forceinline__ unsigned long long box_hash(const double* lo, const double* hi, int verdict) {
    unsigned long long h = 0x9e3779b97f4a7c15ull * (unsigned long long)(verdict + 1);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        h = mix64(h ^ (unsigned long long)__double_as_longlong(lo[d]));
        h = mix64(h + (unsigned long long)__double_as_longlong(hi[d]));
    }
    return h;
}

// Per-block shared state of the level step; WARPS = warps per block.
template <int WARPS>
struct LevelSmem {
    unsigned long long hist[8];
    unsigned long long depth[kDepthBins];
    unsigned long long handles;
    unsigned long long dig_sum, dig_xor;
    // per warp: the lane owning each slot of one iteration's children
    uint8_t own[WARPS][32 * 16];
};

template <int WARPS>
__device__ __forceinline__ void level_smem_init(LevelSmem<WARPS>& sm) {
    for (int t = threadIdx.x; t < kDepthBins; t += blockDim.x) sm.depth[t] = 0;
    if (threadIdx.x < 8) sm.hist[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        sm.handles = 0;
        sm.dig_sum = 0;
        sm.dig_xor = 0;
    }
}

// (defined below)
template <int FAM, int WARPS>
__device__ __forceinline__ void level_emit(const LevelArgs& a, LevelSmem<WARPS>& sm, int v, bool clipped,
                                           bool fp32_decided, const double* lo, const double* hi, int depth,
                                           int given, const LaFree& lf);

// One lane's box j of the chunk (j >= a.count: the lane only takes part in the
// warp's collective child write).  All 32 lanes of the warp must call it.
// ord_in / axis_in >= 0: this box's criterion order / split axis (SPLIT_GIVEN),
// from a network run inline; otherwise the hint arrays (or the defaults).
template <int FAM, int PREC, int WARPS>
__device__ __forceinline__ void level_step(const LevelArgs& a, size_t j, LevelSmem<WARPS>& sm, unsigned& handles,
                                           int ord_in = -1, int axis_in = -1) {
    constexpr int D = family_dims(FAM);
    const size_t i = a.begin + j;
    double lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
    int depth = 0, given = 0;
    int v = -1;                 // this lane's verdict (-1: no box evaluated)
    LaFree lf{0.0, 0.0, 0.0, 0.0};  // start family: the box's lambda-independent terms, when known
    bool clipped = false, fp32_decided = false;
    if (j < a.count) {
        depth = a.in.depth[i];
        if (depth == 0xFF) {
            clipped = true;
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                lo[d] = a.in.lo[d * a.in.cap + i];
                hi[d] = a.in.hi[d * a.in.cap + i];
            }
            const int ord = ord_in >= 0 ? ord_in : (a.order_hint ? a.order_hint[j] : 0);
            LaFree lin{0.0, 0.0, 0.0, 0.0};
            if (FAM == F_START && a.in.aux) {
                lin.flag = a.in.aux[3 * a.in.cap + i];
                if (lin.flag != 0.0) {
                    lin.a13lo = a.in.aux[i];
                    lin.a13hi = a.in.aux[a.in.cap + i];
                    lin.so_hi = a.in.aux[2 * a.in.cap + i];
                }
                lf = lin;
            }
            if (PREC == CP_FP32_PREFILTER) {
                uint8_t pmask;
                const int pre = prefilter_box<FAM>(lo, hi, ord, false, &pmask);
                if (pre == PF_UNDECIDED) {
                    const Verdict r = eval_box<FAM, DECIDE>(lo, hi, ord, nullptr, &lin, &lf);
                    v = r.verdict;
                    handles += r.handles;
                } else {
                    v = pre == PF_PROVED ? V_PROVED : pre == PF_EMPTY ? V_EMPTY : pre == PF_NOFIT ? V_NOFIT : V_CRITICAL;
                    fp32_decided = pre != PF_EMPTY;
                }
            } else {
                const Verdict r = eval_box<FAM, DECIDE>(lo, hi, ord, nullptr, &lin, &lf);
                v = r.verdict;
                handles += r.handles;
            }
            if (a.policy == SPLIT_GIVEN) given = axis_in >= 0 ? axis_in % D : (a.axis_hint ? (a.axis_hint[j] % D) : 0);
        }
    }
    level_emit<FAM>(a, sm, v, clipped, fp32_decided, lo, hi, depth, given, lf);
}

// The end of a level step, for every lane of a warp (all 32 must call it):
// v = the lane's verdict (-1: no box evaluated), its box lo/hi and depth,
// given = its split axis for SPLIT_GIVEN, lf = its lambda-independent terms.
// Counts the verdicts, folds the digest and writes the children of every box
// that is neither proved nor empty (unresolved at the depth limit).
template <int FAM, int WARPS>
__device__ __forceinline__ void level_emit(const LevelArgs& a, LevelSmem<WARPS>& sm, int v, bool clipped,
                                           bool fp32_decided, const double* lo, const double* hi, int depth,
                                           int given, const LaFree& lf) {
    constexpr int D = family_dims(FAM);
    unsigned nchild = 0;
    int axis = 0;
    bool unresolved = false;
    unsigned long long h = 0;  // digest hash of (box, verdict)
    if (v >= 0) {
        if (a.digest) h = box_hash<D>(lo, hi, v);
        if (v != V_PROVED && v != V_EMPTY) {
            if (depth >= a.max_depth) {
                unresolved = true;
            } else {
                nchild = fanout(a.policy, D);
                if (a.policy == SPLIT_WIDEST)
                    axis = widest_axis<D>(lo, hi);
                else if (a.policy == SPLIT_HYBRID)
                    axis = hybrid_axis<D>(lo, hi, a.lambda_scale);
                else if (a.policy == SPLIT_GIVEN)
                    axis = given;
            }
        }
    }
    // counts, once per warp (all 32 lanes are here): one shared-memory atomic
    // per verdict, depth and flag present in the warp instead of one per box
    {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const unsigned b = __ballot_sync(0xffffffffu, v == k);
            if (b && lane == 0) atomicAdd(&sm.hist[k], (unsigned long long)__popc(b));
        }
        const unsigned bc = __ballot_sync(0xffffffffu, clipped);
        const unsigned bu = __ballot_sync(0xffffffffu, unresolved);
        const unsigned bf = __ballot_sync(0xffffffffu, fp32_decided);
        if (lane == 0) {
            if (bc) atomicAdd(&sm.hist[C_CLIPPED], (unsigned long long)__popc(bc));
            if (bu) atomicAdd(&sm.hist[C_UNRESOLVED], (unsigned long long)__popc(bu));
            if (bf) atomicAdd(&sm.hist[C_FP32], (unsigned long long)__popc(bf));
        }
        const int dbin = v >= 0 ? (depth < kDepthBins ? depth : kDepthBins - 1) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, dbin);
        if (dbin >= 0 && lane == __ffs(peers) - 1) atomicAdd(&sm.depth[dbin], (unsigned long long)__popc(peers));
        if (a.digest) {
            unsigned long long hs = v >= 0 ? h : 0ull;
            unsigned long long hx = v >= 0 ? mix64(h ^ 0x5851f42d4c957f2dull) : 0ull;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                hs += __shfl_xor_sync(0xffffffffu, hs, off);
                hx ^= __shfl_xor_sync(0xffffffffu, hx, off);
            }
            if (lane == 0) {
                atomicAdd(&sm.dig_sum, hs);
                atomicXor(&sm.dig_xor, hx);
            }
        }
    }
    // children: the warp reserves one contiguous range and writes it
    // cooperatively, lane k of an iteration writing slot k, so every store
    // of an axis array is one coalesced 256-byte segment per warp
    unsigned excl, total;
    const unsigned long long wbase = warp_reserve_range(&a.cnt[C_OUT], nchild, &excl, &total);
    if (total) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (wbase + total > a.out.cap) {
            if (lane == 0) atomicOr(&a.cnt[C_ERR], E_OVERFLOW);
        } else {
            // slot -> owning lane; the parent box itself comes from the owner by shuffles
            for (unsigned c = 0; c < nchild; ++c) sm.own[w][excl + c] = (uint8_t)lane;
            __syncwarp();
            for (unsigned base = 0; base < total; base += 32) {
                const unsigned k = base + lane;
                const bool valid = k < total;
                const int own = valid ? sm.own[w][k] : 0;
                double plo[4], phi[4], clo[4], chi[4];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    plo[d] = __shfl_sync(0xffffffffu, lo[d], own);
                    phi[d] = __shfl_sync(0xffffffffu, hi[d], own);
                }
                const int c = (int)k - (int)__shfl_sync(0xffffffffu, excl, own);
                const int pax = __shfl_sync(0xffffffffu, axis, own);
                const int pdep = __shfl_sync(0xffffffffu, depth, own);
                LaFree plf{0.0, 0.0, 0.0, 0.0};
                if (FAM == F_START && a.out.aux) {
                    plf.a13lo = __shfl_sync(0xffffffffu, lf.a13lo, own);
                    plf.a13hi = __shfl_sync(0xffffffffu, lf.a13hi, own);
                    plf.so_hi = __shfl_sync(0xffffffffu, lf.so_hi, own);
                    plf.flag = __shfl_sync(0xffffffffu, lf.flag, own);
                }
                if (valid) {
                    make_child<D>(plo, phi, a.policy, pax, c, clo, chi);
                    const bool alive = clip_child<FAM>(clo, chi, a.tab);
                    const size_t o = (size_t)(wbase + k);
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        a.out.lo[d * a.out.cap + o] = clo[d];
                        a.out.hi[d * a.out.cap + o] = chi[d];
                    }
                    a.out.depth[o] = alive ? (uint8_t)(pdep + 1) : (uint8_t)0xFF;
                    if (FAM == F_START && a.out.aux) {
                        // the parent's terms hold for the child when its radii are the parent's, bit for bit
                        bool same = plf.flag != 0.0;
#pragma unroll
                        for (int d = 1; d < D; ++d)
                            same = same && __double_as_longlong(clo[d]) == __double_as_longlong(plo[d]) &&
                                   __double_as_longlong(chi[d]) == __double_as_longlong(phi[d]);
                        a.out.aux[3 * a.out.cap + o] = same ? plf.flag : 0.0;
                        if (same) {
                            a.out.aux[o] = plf.a13lo;
                            a.out.aux[a.out.cap + o] = plf.a13hi;
                            a.out.aux[2 * a.out.cap + o] = plf.so_hi;
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Adds the block's counts to the global counters (after the last step).
template <int WARPS>
__device__ __forceinline__ void level_flush(const LevelArgs& a, LevelSmem<WARPS>& sm, unsigned handles) {
    for (int off = 16; off > 0; off >>= 1) handles += __shfl_xor_sync(0xffffffffu, handles, off);
    if ((threadIdx.x & 31) == 0 && handles) atomicAdd(&sm.handles, (unsigned long long)handles);
    __syncthreads();
    if (threadIdx.x < 8 && threadIdx.x != C_OUT && sm.hist[threadIdx.x])
        atomicAdd(&a.cnt[threadIdx.x], sm.hist[threadIdx.x]);
    if (threadIdx.x == 0 && sm.handles) atomicAdd(&a.cnt[C_HANDLES], sm.handles);
    if (threadIdx.x == 0 && a.digest) {
        atomicAdd(&a.cnt[C_DIGEST], sm.dig_sum);
        atomicXor(&a.cnt[C_DIGEST + 1], sm.dig_xor);
    }
    for (int t = threadIdx.x; t < kDepthBins; t += blockDim.x)
        if (sm.depth[t]) atomicAdd(&a.per_depth[t], sm.depth[t]);
}

}  // namespace cpb

namespace cpb {

// ------------------------------------------------------------------ device-driven loop
// The level-stack schedule of the refinement, kept in device memory so that a
// CUDA graph can run the whole loop without returning to the host.
constexpr int kMaxLevels = 64;

struct DevJob {
    int in_level, out_level;  // out_level < 0: the input level is the last one (no children)
    unsigned long long begin, count;
};

struct DevSched {
    unsigned long long n[kMaxLevels];  // boxes held per level
    DevJob job;                        // the chunk being evaluated
    unsigned long long claim;          // next box of the job handed to a warp
    unsigned long long launches;       // chunks scheduled
    unsigned long long cap;            // boxes per level buffer
    int nlevels, max_depth, fanout;
    int status;                        // 0 ok, 1 worklist capacity exceeded
};

}  // namespace cpb
