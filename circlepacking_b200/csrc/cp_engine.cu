// Prover handle, box refinement (level stack) and the reference-semantics
// lambda loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <queue>
#include <vector>

#include "cp_common.h"
#include "cp_engine.h"
#include "cp_graph_kernels.cuh"
#include "cp_level.cuh"

using namespace cpb;

namespace {

// order-preserving map of a double onto unsigned 64-bit (the encoding of
// Atomic_ordered_double, atomic_float.hpp:56-66)
__host__ __device__ __forceinline__ unsigned long long ordered_bits(double v) {
    unsigned long long b;
    memcpy(&b, &v, 8);
    unsigned long long mask = (0ull - (b >> 63)) | (1ull << 63);
    return b ^ mask;
}
__host__ __device__ __forceinline__ double ordered_value(unsigned long long u) {
    unsigned long long mask = ((u >> 63) - 1) | (1ull << 63);
    unsigned long long b = u ^ mask;
    double v;
    memcpy(&v, &b, 8);
    return v;
}

// MINB: minimum resident blocks per SM requested from the compiler (register cap
// 65536 / (128 * MINB)); the autotuner picks the variant per family and precision.
template <int FAM, int PREC, int MINB>
__global__ void __launch_bounds__(kEvalBlock, MINB) k_level(LevelArgs a) {
    __shared__ LevelSmem<kEvalBlock / 32> sm;
    level_smem_init(sm);
    __syncthreads();
    unsigned handles = 0;
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < a.count; base += step)
        level_step<FAM, PREC>(a, base + threadIdx.x, sm, handles);
    level_flush(a, sm, handles);
}

// Seed: every box of a family lattice, depth 0.
// Lattice seed: box t of this part is lattice box part + t * parts (the lattice
// split into `parts` interleaved pieces; parts = 1: the whole lattice in order).
__global__ void k_seed(LatticeSpec s, const double* __restrict__ slab_single, size_t total, size_t part, size_t parts,
                       BoxList out) {
    const int D = family_dims(s.fam);
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += step) {
        size_t rem = part + t * parts;
        int ix[4] = {0, 0, 0, 0};
        for (int d = D - 1; d >= 0; --d) {
            ix[d] = (int)(rem % (size_t)s.n[d]);
            rem /= (size_t)s.n[d];
        }
        double l[4], h[4];
        const bool visited = lattice_box(s, ix, slab_single[ix[0]], l, h);
        for (int d = 0; d < D; ++d) {
            out.lo[d * out.cap + t] = l[d];
            out.hi[d * out.cap + t] = h[d];
        }
        out.depth[t] = visited ? 0 : 0xFF;
    }
}

__global__ void k_copy_seed(int dims, const double* __restrict__ lo, const double* __restrict__ hi,
                            const uint8_t* __restrict__ depth, size_t n, BoxList out) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += step) {
        for (int d = 0; d < dims; ++d) {
            out.lo[d * out.cap + t] = lo[d * n + t];
            out.hi[d * out.cap + t] = hi[d * n + t];
        }
        out.depth[t] = depth ? depth[t] : 0;
    }
}

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }
__global__ void k_zero_u64(unsigned long long* p, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0;
}

// The graph engine's level table and schedule, passed by value (about 3 KB of
// kernel parameters).
struct GraphUpload {
    BoxList levels[kMaxLevels];
    DevSched sched;
    int nlevels;
};
__global__ void k_graph_upload(GraphUpload u, BoxList* levels, DevSched* sched) {
    for (int l = threadIdx.x; l < u.nlevels; l += blockDim.x) levels[l] = u.levels[l];
    if (threadIdx.x == 0) *sched = u.sched;
}

// Seeded random boxes on the family's domain (the uneven-depth workload of the
// persistent engine).  Box i draws its numbers from a counter-based generator:
// u(i, k) = top 53 bits of mix64(seed ^ mix64(8 i + k)) / 2^53.  Lambda has its
// centre uniform in [0.5, 0.99]; each radius has its centre uniform in the
// dependent range of the axes before it (the ranges the lattice enumerates,
// with the single-placement table's upper bound); every axis has a log-uniform
// width in [2^-20, 2^-4] and is intersected with its range.  A box whose range
// is empty is marked dropped (depth 0xFF); the others get a depth label
// uniform in 0..max_label.
__device__ __forceinline__ double rand_unit(unsigned long long seed, unsigned long long i, int k) {
    const unsigned long long z = mix64(seed ^ mix64(8ull * i + (unsigned long long)k));
    return (double)(z >> 11) * 0x1.0p-53;
}
__device__ __forceinline__ bool rand_axis(unsigned long long seed, unsigned long long i, int k, Iv range, double* lo,
                                          double* hi) {
    if (!(range.lo <= range.hi)) return false;
    const double c = range.lo + (range.hi - range.lo) * rand_unit(seed, i, k);
    const double w = exp2(-20.0 + 16.0 * rand_unit(seed, i, k + 1));
    *lo = fmax(range.lo, c - 0.5 * w);
    *hi = fmin(range.hi, c + 0.5 * w);
    return *lo <= *hi;
}
__global__ void k_random_boxes(int fam, unsigned long long seed, int max_label, size_t n, SingleTable tab, BoxList out) {
    const int D = family_dims(fam);
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += step) {
        double l[4] = {0, 0, 0, 0}, h[4] = {0, 0, 0, 0};
        bool alive = rand_axis(seed, t, 0, Iv{kLambdaMin, kLambdaMax}, &l[0], &h[0]);
        const Iv la{l[0], h[0]};
        if (alive) alive = rand_axis(seed, t, 2, range_r1(la, single_upper(tab, la.lo)), &l[1], &h[1]);
        if (alive) alive = rand_axis(seed, t, 4, range_r2(fam, la, Iv{l[1], h[1]}), &l[2], &h[2]);
        if (alive && D == 4) alive = rand_axis(seed, t, 6, range_r3(fam, la, Iv{l[2], h[2]}), &l[3], &h[3]);
        for (int d = 0; d < D; ++d) {
            out.lo[d * out.cap + t] = l[d];
            out.hi[d * out.cap + t] = h[d];
        }
        const int label = (int)(rand_unit(seed, t, 8) * (double)(max_label + 1));
        out.depth[t] = alive ? (uint8_t)(label > max_label ? max_label : label) : (uint8_t)0xFF;
    }
}

__global__ void k_single_table(double lo, double h, int n, double* t, double* v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = __fma_rn((double)i, h, lo);
        t[i] = x;
        v[i] = single_placement(x);
    }
}

// The device-side scheduler of the graph-driven loop (one thread): commits the
// previous chunk (input consumed, children appended), then picks the next
// chunk exactly as the host loop does -- the deepest non-empty level, as many
// boxes as the next level has room for -- or ends the loop.
constexpr unsigned long long kGraphLaunchLimit = 1ull << 22;
__global__ void k_sched(DevSched* s, unsigned long long* cnt, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    DevJob& j = s->job;
    if (j.count) {
        s->n[j.in_level] -= j.count;
        if (j.out_level >= 0) s->n[j.out_level] = cnt[C_OUT];
        j.count = 0;
        if (cnt[C_ERR] & E_OVERFLOW) {
            s->status = 1;
            cudaGraphSetConditional(h, 0);
            return;
        }
    }
    int l = -1;
    for (int k = s->nlevels - 1; k >= 0; --k)
        if (s->n[k]) {
            l = k;
            break;
        }
    if (l < 0) {
        cudaGraphSetConditional(h, 0);
        return;
    }
    if (s->launches >= kGraphLaunchLimit) {  // bound on the loop (cannot be reached by a valid schedule)
        s->status = 2;
        cudaGraphSetConditional(h, 0);
        return;
    }
    const int out = (l + 1 < s->nlevels && l < s->max_depth) ? l + 1 : -1;
    unsigned long long c = s->n[l];
    if (out >= 0) {
        const unsigned long long room = (s->cap - s->n[out]) / (unsigned long long)s->fanout;
        if (room < c) c = room;
        if (c == 0) {
            s->status = 1;
            cudaGraphSetConditional(h, 0);
            return;
        }
    }
    j.in_level = l;
    j.out_level = out;
    j.begin = s->n[l] - c;
    j.count = c;
    cnt[C_OUT] = out >= 0 ? s->n[out] : 0;
    s->claim = 0;
    s->launches += 1;
}

// ------------------------------------------------------------------ reference step
struct RefArgs {
    LatticeSpec s;
    const double* slab_single;
    int slab_begin;
    size_t count;  // boxes in this wave
    unsigned long long* cnt;
    int collect;  // 1: record every failing box (no early exit)
    double* coll;
    uint8_t* coll_handles;
    size_t coll_cap;
};

// The body of the family kernels' loops (e.g. middle_configuration.cu:157-201)
// over the lattice boxes of lambda slabs [slab_begin, ...), stopping at slabs
// beyond the first slab that holds a failing box.
template <int FAM>
__global__ void __launch_bounds__(kEvalBlock) k_ref_step(RefArgs a) {
    constexpr int D = family_dims(FAM);
    size_t per_slab = 1;
    for (int d = 1; d < D; ++d) per_slab *= (size_t)a.s.n[d];
    const size_t step = (size_t)gridDim.x * blockDim.x;
    unsigned long long evaluated = 0;
    volatile unsigned long long* best = a.cnt + C_BEST_SLAB;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.count; t += step) {
        const int slab = a.slab_begin + (int)(t / per_slab);
        if (!a.collect && (unsigned long long)slab > *best) continue;
        size_t rem = t % per_slab;
        int ix[4] = {slab, 0, 0, 0};
        for (int d = D - 1; d >= 1; --d) {
            ix[d] = (int)(rem % (size_t)a.s.n[d]);
            rem /= (size_t)a.s.n[d];
        }
        double lo[4], hi[4];
        if (!lattice_box(a.s, ix, a.slab_single[slab], lo, hi)) continue;
        ++evaluated;
        Verdict v = a.collect ? eval_box<FAM, FULL>(lo, hi, 0, nullptr) : eval_box<FAM, DECIDE>(lo, hi, 0, nullptr);
        if (v.verdict == V_EMPTY) continue;
        const bool nofit = (v.mask & M_FIT) && FAM != F_START && FAM != F_START_END_2D && FAM != F_START_END_3D;
        const bool trap = (v.mask & M_TRAP) != 0;
        if (nofit || trap) {
            atomicMin(&a.cnt[trap ? C_TRAP_SLAB : C_NOFIT_SLAB], (unsigned long long)slab);
            if (atomicCAS(&a.cnt[C_ERRBOX_CLAIM], 0ull, 1ull) == 0ull) {
                for (int d = 0; d < D; ++d) {
                    a.cnt[C_ERRBOX + 2 * d] = __double_as_longlong(lo[d]);
                    a.cnt[C_ERRBOX + 2 * d + 1] = __double_as_longlong(hi[d]);
                }
            }
        }
        if (v.mask & M_CRIT) {
            atomicMin(&a.cnt[C_BEST_SLAB], (unsigned long long)slab);
            atomicMin(&a.cnt[C_FIRST_BITS], ordered_bits(lo[0]));
            if (a.collect) {
                const unsigned long long k = atomicAdd(&a.cnt[C_COLLECT], 1ull);
                if (k < a.coll_cap) {
                    // the box as the reference prints it: r2, r1 tightened
                    if (D == 4 && lo[2] < lo[3]) lo[2] = lo[3];
                    if (lo[1] < lo[2]) lo[1] = lo[2];
                    double* rec = a.coll + 8 * k;
                    for (int d = 0; d < 4; ++d) {
                        rec[2 * d] = d < D ? lo[d] : 0.0;
                        rec[2 * d + 1] = d < D ? hi[d] : 0.0;
                    }
                    uint8_t hb = v.mask & M_CRIT;
                    if (FAM == F_MIDDLE) hb = (uint8_t)(((hb & 3) ? 1 : 0) | ((hb & 12) ? 2 : 0));
                    a.coll_handles[k] = hb;
                }
            }
        }
    }
    if (evaluated) atomicAdd(&a.cnt[C_EVALUATED], evaluated);
}

template <class K>
unsigned grid_of(K kernel, int block) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return (unsigned)(sms * per_sm);
}

constexpr double kDefaultLambdaScale = 4e-3;
double lambda_scale_of(const cp_refine_opts& o) { return o.lambda_scale > 0.0 ? o.lambda_scale : kDefaultLambdaScale; }

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ------------------------------------------------------------------ handle
struct LevelBuf {
    BoxList b{nullptr, nullptr, nullptr, 0, nullptr};
    size_t n = 0;
    double* aux = nullptr;  // kAuxFields x cap, allocated on first use (b.aux points here when in use)
};

struct cp_prover {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::atomic<int> interrupt{0};
    unsigned long long* cnt = nullptr;  // C_COUNT counters
    unsigned long long* per_depth = nullptr;
    unsigned long long* h_cnt = nullptr;  // pinned mirror
    double* tab_t = nullptr;
    double* tab_v = nullptr;
    int tab_n = 0;
    double tab_h = 0;
    double* slab_single = nullptr;
    int slab_cap = 0;
    std::vector<LevelBuf> levels;
    int levels_dims = 0;
    size_t level_cap = 0;
    void* model = nullptr;  // learned model state (cp_model.cu)
    // device-driven loop (CUDA graph with a conditional WHILE node)
    BoxList* d_levels = nullptr;
    DevSched* d_sched = nullptr;
    DevSched* h_sched = nullptr;  // pinned mirror
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    unsigned long long graph_key[12] = {0};
    int graph_variant[6][2] = {{1, 1}, {1, 1}, {1, 1}, {1, 1}, {1, 1}, {1, 1}};  // block-size variant
    int graph_bpt[6][2] = {{2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}, {2, 2}};      // boxes per thread
    // an interrupted host-driven refinement: the level stack and counters hold
    // its remaining boxes and partial counts (cp_refine_resume, checkpoints)
    bool pending = false;
    cp_refine_opts pending_opts{};
    int variant[6][2] = {{1, 1}, {0, 0}, {1, 1}, {1, 1}, {0, 0}, {1, 1}};  // level-kernel variant per family/precision
    // called before every lattice launch of cp_prove_family_reference
    cp_step_callback step_cb = nullptr;
    void* step_user = nullptr;
    // called after every chunk of a host-driven refinement
    cp_chunk_callback chunk_cb = nullptr;
    void* chunk_user = nullptr;
    // host seeds staged on a copy stream (cp_stage_boxes_host / cp_refine_staged)
    cudaStream_t copy_stream = nullptr;
    struct Stage {
        unsigned char* buf = nullptr;  // lo [dims][n] doubles, hi [dims][n] doubles, depth [n] bytes
        size_t bytes = 0, n = 0;
        int dims = 0;
        bool has_depth = false, staged = false;
        cudaEvent_t done = nullptr;  // the copy has landed
    } stage[2];
};

cudaStream_t cp_prover_stream(cp_prover* p) { return p->stream; }
void*& cp_prover_model(cp_prover* p) { return p->model; }

namespace {

cp_status cuda_ok(cudaError_t e, cp_status s = CP_ERR_CUDA) {
    if (e == cudaSuccess) return CP_OK;
    return cp_record_cuda_error(e, e == cudaErrorMemoryAllocation ? CP_ERR_NOMEM : s);
}
#define CP_TRY(x)                      \
    do {                               \
        cp_status s_ = (x);            \
        if (s_ != CP_OK) return s_;    \
    } while (0)

// Zeroes the counters and per-depth bins with a kernel: a memset may run on a
// copy engine and wait there behind a large host-to-device copy of staged seeds.
cp_status reset_counters(cp_prover* p) {
    k_zero_u64<<<1, 128, 0, p->stream>>>(p->cnt, (int)(C_COUNT + kDepthBins));
    return cp_check_launch();
}

cp_status read_counters(cp_prover* p) {
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->h_cnt, p->cnt, sizeof(unsigned long long) * (C_COUNT + kDepthBins),
                                   cudaMemcpyDeviceToHost, p->stream)));
    return cuda_ok(cudaStreamSynchronize(p->stream));
}

void free_levels(cp_prover* p) {
    for (auto& L : p->levels) {
        cudaFree(L.b.lo);
        cudaFree(L.b.hi);
        cudaFree(L.b.depth);
        cudaFree(L.aux);
    }
    p->levels.clear();
}

cp_status ensure_levels(cp_prover* p, int count, int dims, size_t cap) {
    if ((int)p->levels.size() >= count && p->levels_dims >= dims && p->level_cap == cap) return CP_OK;
    if (p->levels_dims < dims || p->level_cap != cap) free_levels(p);
    p->levels_dims = dims;
    p->level_cap = cap;
    while ((int)p->levels.size() < count) {
        LevelBuf L;
        L.b.cap = cap;
        CP_TRY(cuda_ok(cudaMalloc(&L.b.lo, sizeof(double) * dims * cap)));
        CP_TRY(cuda_ok(cudaMalloc(&L.b.hi, sizeof(double) * dims * cap)));
        CP_TRY(cuda_ok(cudaMalloc(&L.b.depth, cap)));
        p->levels.push_back(L);
    }
    return CP_OK;
}

cp_status ensure_slab(cp_prover* p, int n) {
    if (p->slab_cap >= n) return CP_OK;
    cudaFree(p->slab_single);
    p->slab_single = nullptr;
    p->slab_cap = 0;
    CP_TRY(cuda_ok(cudaMalloc(&p->slab_single, sizeof(double) * n)));
    p->slab_cap = n;
    return CP_OK;
}

SingleTable table_of(const cp_prover* p) { return SingleTable{p->tab_t, p->tab_v, p->tab_n, p->tab_h}; }

using LevelKernel = void (*)(LevelArgs);
// register variants of the level kernel: minimum resident blocks 1, 4, 5, 6
constexpr int kVariants = 4;
template <int FAM, int PREC>
LevelKernel level_variant(int v) {
    switch (v) {
    case 1: return k_level<FAM, PREC, 4>;
    case 2: return k_level<FAM, PREC, 5>;
    case 3: return k_level<FAM, PREC, 6>;
    default: return k_level<FAM, PREC, 1>;
    }
}
template <int FAM>
LevelKernel level_variant_p(int prec, int v) {
    return prec ? level_variant<FAM, 1>(v) : level_variant<FAM, 0>(v);
}
LevelKernel level_kernel(int fam, int prec, int v) {
    switch (fam) {
    case 0: return level_variant_p<0>(prec, v);
    case 1: return level_variant_p<1>(prec, v);
    case 2: return level_variant_p<2>(prec, v);
    case 3: return level_variant_p<3>(prec, v);
    case 4: return level_variant_p<4>(prec, v);
    default: return level_variant_p<5>(prec, v);
    }
}

using RefKernel = void (*)(RefArgs);
RefKernel ref_kernel(int fam) {
    static const RefKernel k[6] = {k_ref_step<0>, k_ref_step<1>, k_ref_step<2>,
                                   k_ref_step<3>, k_ref_step<4>, k_ref_step<5>};
    return k[fam];
}

// the reference's lattice sizes per family (start_configuration.cu:41-53,
// middle_configuration.cu:39-42, end_configuration.cu:39-49)
void reference_sizes(int fam, int* n) {
    static const int s[6][4] = {{256, 256, 256, 64}, {4096, 4096, 4096, 1}, {256, 256, 256, 64},
                                {512, 256, 256, 64}, {4096, 1024, 1024, 1}, {1024, 256, 128, 128}};
    for (int d = 0; d < 4; ++d) n[d] = s[fam][d];
}

}  // namespace

// ------------------------------------------------------------------ engine pieces
size_t cp_engine_counter_words() { return (size_t)(C_COUNT + kDepthBins); }

cp_status cp_engine_launch_table(double lambda_lo, double h, int n, double* t, double* v, cudaStream_t st) {
    k_single_table<<<64, 128, 0, st>>>(lambda_lo, h, n, t, v);
    return cp_check_launch();
}

cp_status cp_engine_launch_level(int fam, int prec, int variant, const BoxList& in, size_t begin, size_t count,
                                 const BoxList* out, unsigned long long out_base, unsigned long long* counters,
                                 const double* tab_t, const double* tab_v, int tab_n, double tab_h, int policy,
                                 int max_depth, cudaStream_t st) {
    LevelArgs a;
    a.in = in;
    a.begin = begin;
    a.count = count;
    a.out = out ? *out : BoxList{nullptr, nullptr, nullptr, 0};
    a.cnt = counters;
    a.per_depth = counters + C_COUNT;
    a.tab = SingleTable{tab_t, tab_v, tab_n, tab_h};
    a.policy = policy == CP_SPLIT_LEARNED ? SPLIT_GIVEN : policy;
    a.lambda_scale = kDefaultLambdaScale;
    a.max_depth = out ? max_depth : 0;
    a.axis_hint = nullptr;
    a.order_hint = nullptr;
    a.digest = 0;
    cudaError_t e = cudaMemcpyAsync(counters + C_OUT, &out_base, sizeof(out_base), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    LevelKernel k = level_kernel(fam, prec, variant);
    const int block = kEvalBlock;
    unsigned grid = grid_of(k, block);
    const size_t need = (count + block - 1) / block;
    if (need < grid) grid = (unsigned)std::max<size_t>(need, 1);
    k<<<grid, block, 0, st>>>(a);
    return cp_check_launch();
}

bool cp_engine_overflowed(const unsigned long long* h) { return (h[C_ERR] & E_OVERFLOW) != 0; }
unsigned long long cp_engine_children(const unsigned long long* h) { return h[C_OUT]; }

void cp_engine_fill_report(const unsigned long long* h, cp_refine_report* r) {
    for (int v = 0; v < 5; ++v) r->verdicts[v] = (int64_t)h[C_VERDICT + v];
    r->unresolved = (int64_t)h[C_UNRESOLVED];
    r->clipped = (int64_t)h[C_CLIPPED];
    r->fp32_decided = (int64_t)h[C_FP32];
    r->handles_evaluated = (int64_t)h[C_HANDLES];
    r->digest[0] = (uint64_t)h[C_DIGEST];
    r->digest[1] = (uint64_t)h[C_DIGEST + 1];
    r->evaluated = 0;
    for (int v = 0; v < 5; ++v) r->evaluated += r->verdicts[v];
    r->max_depth_seen = 0;
    for (int d = 0; d < kDepthBins; ++d) {
        r->per_depth[d] = (int64_t)h[C_COUNT + d];
        if (r->per_depth[d]) r->max_depth_seen = d;
    }
}

// ------------------------------------------------------------------ internal API
cp_status cp_engine_eval_chunk(cp_prover* p, int fam, const cp_refine_opts& o, LevelBuf& in, size_t begin,
                               size_t count, LevelBuf* out, const uint8_t* axis_hint, const uint8_t* order_hint,
                               double* ms) {
    LevelArgs a;
    a.in = in.b;
    a.begin = begin;
    a.count = count;
    a.out = out ? out->b : BoxList{nullptr, nullptr, nullptr, 0};
    a.cnt = p->cnt;
    a.per_depth = p->per_depth;
    a.tab = table_of(p);
    a.policy = o.policy == CP_SPLIT_LEARNED ? SPLIT_GIVEN : o.policy;
    a.lambda_scale = lambda_scale_of(o);
    a.max_depth = out ? o.max_depth : 0;
    a.axis_hint = axis_hint;
    a.order_hint = order_hint;
    a.digest = o.digest ? 1 : 0;
    // children append after the boxes already in `out`
    unsigned long long base = out ? out->n : 0;
    k_set_u64<<<1, 1, 0, p->stream>>>(p->cnt + C_OUT, base);
    CP_TRY(cp_check_launch());
    LevelKernel k = level_kernel(fam, o.precision, p->variant[fam][o.precision ? 1 : 0]);
    const int block = kEvalBlock;
    unsigned grid = grid_of(k, block);
    size_t need = (count + block - 1) / block;
    if (need < grid) grid = (unsigned)std::max<size_t>(need, 1);
    cudaEventRecord(p->ev0, p->stream);
    k<<<grid, block, 0, p->stream>>>(a);
    cudaEventRecord(p->ev1, p->stream);
    CP_TRY(cp_check_launch());
    CP_TRY(read_counters(p));
    float t = 0;
    cudaEventElapsedTime(&t, p->ev0, p->ev1);
    *ms += t;
    if (p->h_cnt[C_ERR] & E_OVERFLOW) return CP_ERR_CAPACITY;
    if (out) out->n = (size_t)p->h_cnt[C_OUT];
    return CP_OK;
}

namespace {

cp_status refine_levels(cp_prover* p, const cp_refine_opts& o, cp_refine_report* r, double t_wall0) {
    const int fam = o.family;
    const int D = family_dims(fam);
    const int F = fanout(o.policy == CP_SPLIT_LEARNED ? SPLIT_GIVEN : o.policy, D);
    double ms = 0;
    int launches = 0;
    const int L = o.max_depth;
    for (;;) {
        int l = -1;
        for (int k = (int)p->levels.size() - 1; k >= 0; --k)
            if (p->levels[k].n > 0) {
                l = k;
                break;
            }
        if (l < 0) break;
        LevelBuf& in = p->levels[l];
        LevelBuf* out = (l + 1 < (int)p->levels.size() && l < L) ? &p->levels[l + 1] : nullptr;
        size_t c;
        if (out) {
            size_t free_slots = out->b.cap - out->n;
            c = std::min(in.n, free_slots / (size_t)F);
            if (c == 0) return CP_ERR_CAPACITY;
        } else {
            c = in.n;
        }
        const size_t begin = in.n - c;
        uint8_t *axis = nullptr, *order = nullptr;
        if (cp_model_collecting(p))
            CP_TRY(cp_model_collect_chunk(p, fam, in.b, begin, c, p->tab_t, p->tab_v, p->tab_n, p->tab_h));
        if (o.policy == CP_SPLIT_LEARNED || o.learned_order) {
            // the inference launch is part of the refinement's device time
            CP_TRY(cuda_ok(cudaEventRecord(p->ev0, p->stream)));
            CP_TRY(cp_model_hints(p, fam, in.b, begin, c, o.policy == CP_SPLIT_LEARNED ? &axis : nullptr,
                                  o.learned_order ? &order : nullptr));
            CP_TRY(cuda_ok(cudaEventRecord(p->ev1, p->stream)));
            CP_TRY(cuda_ok(cudaEventSynchronize(p->ev1)));
            float t = 0;
            cudaEventElapsedTime(&t, p->ev0, p->ev1);
            ms += t;
        }
        CP_TRY(cp_engine_eval_chunk(p, fam, o, in, begin, c, out, axis, order, &ms));
        ++launches;
        in.n -= c;
        if (p->chunk_cb) {
            int64_t evaluated = 0, waiting = 0;
            for (int v = 0; v < 5; ++v) evaluated += (int64_t)p->h_cnt[C_VERDICT + v];
            for (const auto& L : p->levels) waiting += (int64_t)L.n;
            p->chunk_cb(p->chunk_user, evaluated, waiting);
        }
        if (p->interrupt.load()) {
            p->interrupt.store(0);
            p->pending = true;
            p->pending_opts = o;
            return CP_ERR_INTERRUPTED;
        }
    }
    (void)D;
    cp_engine_fill_report(p->h_cnt, r);
    r->launches = launches;
    r->device_ms = ms;
    r->wall_ms = now_ms() - t_wall0;
    return CP_OK;
}

void free_graph(cp_prover* p) {
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->graph_exec = nullptr;
    p->graph = nullptr;
    std::memset(p->graph_key, 0, sizeof(p->graph_key));
}

int graph_variant_of_block(int block) {
    for (int v = 0; v < kGraphVariants; ++v)
        if (kGraphBlock[v] == block) return v;
    return -1;
}

// Builds the graph of the device-driven loop: a WHILE node whose body is
// scheduler -> (model hints) -> persistent level kernel.
cp_status build_graph(cp_prover* p, const cp_refine_opts& o, int variant, int bpt, bool learned_axis,
                      bool learned_order) {
    free_graph(p);
    const int fam = o.family;
    const int prec = o.precision ? 1 : 0;
    CP_TRY(cuda_ok(cudaGraphCreate(&p->graph, 0)));
    cudaGraphConditionalHandle h;
    CP_TRY(cuda_ok(cudaGraphConditionalHandleCreate(&h, p->graph, 1, cudaGraphCondAssignDefault)));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CP_TRY(cuda_ok(cudaGraphAddNode(&node, p->graph, nullptr, 0, &cp)));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CP_TRY(cuda_ok(cudaStreamBeginCaptureToGraph(p->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)));
    cp_status st = CP_OK;
    do {
        k_sched<<<1, 32, 0, p->stream>>>(p->d_sched, p->cnt, h);
        if ((st = cp_check_launch()) != CP_OK) break;
        // with a learned policy the level kernel runs the network inline (tcgen05)
        const bool net = learned_axis || learned_order;
        NetArgs na{};
        if (net) {
            const void* views = nullptr;
            const float* master = nullptr;
            int limit = 0;
            if ((st = cp_model_net_params(p, fam, &views, &master, &limit)) != CP_OK) break;
            na.views = static_cast<const tc::bf16*>(views);
            na.master = master;
            na.wait_limit = limit;
            na.want_order = learned_order ? 1 : 0;
            na.want_axis = learned_axis ? 1 : 0;
        }
        PersistArgs pa;
        pa.levels = p->d_levels;
        pa.sched = p->d_sched;
        pa.cnt = p->cnt;
        pa.per_depth = p->per_depth;
        pa.tab = table_of(p);
        pa.policy = o.policy == CP_SPLIT_LEARNED ? SPLIT_GIVEN : o.policy;
        pa.lambda_scale = lambda_scale_of(o);
        pa.max_depth = o.max_depth;
        pa.bpt = bpt;
        pa.axis_hint = nullptr;
        pa.order_hint = nullptr;
        pa.digest = o.digest ? 1 : 0;
        void* kern = net ? (prec ? cp_graph_kernel_net_fp32(fam) : cp_graph_kernel_net_fp64(fam))
                         : (prec ? cp_graph_kernel_fp32(fam, variant) : cp_graph_kernel_fp64(fam, variant));
        const int block = net ? kNetBlock : kGraphBlock[variant];
        int per_sm = 0, sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
        if (net) {
            // The occupancy calculator reports one CTA per SM for the kernel that
            // uses tensor memory, while the SM keeps as many resident as its
            // registers, shared memory (about 32 KB per CTA, largest carveout)
            // and tensor memory (tc::kNetCols columns per CTA) allow; the grid is
            // sized from those limits.  A CTA beyond the resident ones starts when
            // one ends (the kernel claims work dynamically), so an overestimate
            // costs a few idle CTAs, never a wait on one another.
            cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
            cudaFuncAttributes fa{};
            int regs_sm = 65536, smem_sm = 0;
            cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, p->device);
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, p->device);
            if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess && fa.numRegs > 0) {
                const int by_regs = regs_sm / (((fa.numRegs + 7) / 8 * 8) * block);
                const int by_smem = smem_sm / ((int)fa.sharedSizeBytes + 1024);  // 1 KB reserved per CTA
                per_sm = std::min(std::min(by_regs, by_smem), kNetMaxCtasPerSm);
            }
            if (per_sm < 1) per_sm = 1;
        } else if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0) != cudaSuccess || per_sm < 1) {
            per_sm = 1;
        }
        void* args[] = {&pa};
        void* net_args[] = {&pa, &na};
        st = cuda_ok(cudaLaunchKernel(kern, dim3((unsigned)(sms * per_sm)), dim3((unsigned)block), net ? net_args : args,
                                      0, p->stream));
    } while (0);
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(p->stream, &captured);
    if (st != CP_OK) return st;
    CP_TRY(cuda_ok(ec));
    return cuda_ok(cudaGraphInstantiate(&p->graph_exec, p->graph, 0));
}

// The level-stack loop of refine_levels, run on the device by one CUDA graph
// launch: no host round trip between chunks.
cp_status refine_graph(cp_prover* p, const cp_refine_opts& o, cp_refine_report* r, double t_wall0) {
    const int fam = o.family;
    const int D = family_dims(fam);
    const int prec = o.precision ? 1 : 0;
    const int nlevels = (int)p->levels.size();
    if (nlevels > kMaxLevels) return cp_fail(CP_ERR_INVALID, "graph engine: max_depth must be < %d", kMaxLevels);
    int variant = o.block > 0 ? graph_variant_of_block(o.block) : p->graph_variant[fam][prec];
    if (variant < 0) return cp_fail(CP_ERR_INVALID, "graph engine: block must be 64, 128, 256, 512 or 1024");
    const int bpt = o.boxes_per_thread > 0 ? o.boxes_per_thread : p->graph_bpt[fam][prec];
    if (bpt > 8) return cp_fail(CP_ERR_INVALID, "graph engine: boxes_per_thread must be 1..8");
    const bool learned_axis = o.policy == CP_SPLIT_LEARNED, learned_order = o.learned_order != 0;
    if (!p->d_levels) {
        CP_TRY(cuda_ok(cudaMalloc(&p->d_levels, sizeof(BoxList) * kMaxLevels)));
        CP_TRY(cuda_ok(cudaMalloc(&p->d_sched, sizeof(DevSched))));
        CP_TRY(cuda_ok(cudaMallocHost(&p->h_sched, sizeof(DevSched))));
    }
    BoxList hl[kMaxLevels];
    for (int l = 0; l < nlevels; ++l) hl[l] = p->levels[l].b;
    DevSched& hs = *p->h_sched;
    std::memset(&hs, 0, sizeof(hs));
    for (int l = 0; l < nlevels; ++l) hs.n[l] = p->levels[l].n;
    hs.cap = p->level_cap;
    hs.nlevels = nlevels;
    hs.max_depth = o.max_depth;
    hs.fanout = fanout(o.policy == CP_SPLIT_LEARNED ? SPLIT_GIVEN : o.policy, D);
    {
        // the level table and the schedule travel as kernel parameters: a copy
        // would queue behind a large host-to-device copy of staged seeds on the
        // copy engine and delay the refinement
        GraphUpload u;
        for (int l = 0; l < nlevels; ++l) u.levels[l] = hl[l];
        u.sched = hs;
        u.nlevels = nlevels;
        k_graph_upload<<<1, 64, 0, p->stream>>>(u, p->d_levels, p->d_sched);
        CP_TRY(cp_check_launch());
    }
    double ls = lambda_scale_of(o);
    unsigned long long ls_bits;
    std::memcpy(&ls_bits, &ls, 8);
    const unsigned long long key[12] = {ls_bits, (unsigned long long)fam + 1, (unsigned long long)prec, (unsigned long long)variant,
                                        (unsigned long long)bpt, (unsigned long long)o.policy,
                                        (unsigned long long)o.max_depth,
                                        (unsigned long long)(learned_axis | (learned_order << 1) | (o.digest ? 4 : 0)),
                                        (unsigned long long)(uintptr_t)p->levels[0].b.lo, (unsigned long long)p->level_cap,
                                        (unsigned long long)nlevels,
                                        (unsigned long long)(uintptr_t)p->model};
    if (!p->graph_exec || std::memcmp(key, p->graph_key, sizeof(key)) != 0) {
        CP_TRY(build_graph(p, o, variant, bpt, learned_axis, learned_order));
        std::memcpy(p->graph_key, key, sizeof(key));
    }
    CP_TRY(cuda_ok(cudaEventRecord(p->ev0, p->stream)));
    CP_TRY(cuda_ok(cudaGraphLaunch(p->graph_exec, p->stream)));
    CP_TRY(cuda_ok(cudaEventRecord(p->ev1, p->stream)));
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->h_sched, p->d_sched, sizeof(DevSched), cudaMemcpyDeviceToHost, p->stream)));
    CP_TRY(read_counters(p));
    float t = 0;
    cudaEventElapsedTime(&t, p->ev0, p->ev1);
    for (int l = 0; l < nlevels; ++l) p->levels[l].n = (size_t)p->h_sched->n[l];
    if (p->h_sched->status == 1) return cp_fail(CP_ERR_CAPACITY, "graph engine: worklist level capacity exceeded");
    if (p->h_cnt[C_ERR] & E_TC)
        return cp_fail(CP_ERR_DEVICE, "graph engine: a tensor-core completion wait of the inline network timed out");
    if (p->h_sched->status != 0) return cp_fail(CP_ERR_DEVICE, "graph engine: scheduler stopped (status %d)",
                                                p->h_sched->status);
    cp_engine_fill_report(p->h_cnt, r);
    r->launches = (int32_t)p->h_sched->launches;
    r->device_ms = t;
    r->wall_ms = now_ms() - t_wall0;
    return CP_OK;
}

// The lambda-independent terms of the start family travel with the boxes of
// levels >= 1 (children) when the refinement asks for it (opts.reuse) and its
// split can leave radii unchanged; every other refinement, and the seed level,
// sees no aux.  A level whose aux cannot be allocated goes without: its boxes
// recompute the terms.
void attach_aux(cp_prover* p, const cp_refine_opts& o) {
    // a uniform split changes every radius of every child: nothing to carry
    const bool use = o.reuse != 0 && o.family == F_START && o.policy != CP_SPLIT_UNIFORM;
    for (size_t l = 0; l < p->levels.size(); ++l) {
        LevelBuf& L = p->levels[l];
        if (use && l > 0 && !L.aux && cudaMalloc(&L.aux, sizeof(double) * kAuxFields * L.b.cap) != cudaSuccess) {
            L.aux = nullptr;
            cudaGetLastError();  // clear the allocation error
        }
        L.b.aux = (use && l > 0) ? L.aux : nullptr;
    }
}

cp_status run_refinement(cp_prover* p, const cp_refine_opts& o, cp_refine_report* r, double t0) {
    attach_aux(p, o);
    if (o.engine == CP_ENGINE_GRAPH && !cp_model_collecting(p)) return refine_graph(p, o, r, t0);
    return refine_levels(p, o, r, t0);
}

// lower end of seed slab k of a proof (slab k covers [cut(k), cut(k + 1)])
double proof_slab_cut(const cp_proof_opts& o, int k) {
    if (k <= 0) return kLambdaMin;
    if (k >= o.slabs) return kLambdaMax;
    if (!o.geometric) return kLambdaMin + (kLambdaMax - kLambdaMin) / o.slabs * k;
    // 1 - lambda from 0.5 down to 0.01 by a constant factor per slab
    return 1.0 - (1.0 - kLambdaMin) * std::pow((1.0 - kLambdaMax) / (1.0 - kLambdaMin), (double)k / o.slabs);
}

cp_status check_opts(const cp_refine_opts* o) {
    if (!o || o->family < 0 || o->family > 5) return CP_ERR_INVALID;
    if (o->precision != CP_FP64 && o->precision != CP_FP32_PREFILTER) return CP_ERR_INVALID;
    if (o->policy < CP_SPLIT_UNIFORM || o->policy > CP_SPLIT_HYBRID) return CP_ERR_INVALID;
    if (!(o->lambda_scale >= 0.0)) return CP_ERR_INVALID;
    if (o->max_depth < 0 || o->max_depth > 250) return CP_ERR_INVALID;
    if (o->engine != CP_ENGINE_LEVELS && o->engine != CP_ENGINE_GRAPH) return CP_ERR_INVALID;
    if (o->boxes_per_thread < 0 || o->boxes_per_thread > 8) return CP_ERR_INVALID;
    if (o->seed_parts < 0 || (o->seed_parts > 1 && (o->seed_part < 0 || o->seed_part >= o->seed_parts)))
        return CP_ERR_INVALID;
    return CP_OK;
}

}  // namespace

// cp_refine without clearing a pending interrupt request (internal: not exported)
extern "C" __attribute__((visibility("hidden"))) cp_status cp_refine_keep_interrupt(cp_prover* p,
                                                                                      const cp_refine_opts* o,
                                                                                      cp_refine_report* r);


extern "C" {

cp_status cp_create(int device, cp_prover** out) {
    if (!out) return CP_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return CP_ERR_NO_DEVICE;
    }
    CP_TRY(cuda_ok(cudaSetDevice(device)));
    cp_prover* p = new cp_prover();
    p->device = device;
    cp_status s = CP_OK;
    do {
        if ((s = cuda_ok(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking))) != CP_OK) break;
        if ((s = cuda_ok(cudaEventCreate(&p->ev0))) != CP_OK) break;
        if ((s = cuda_ok(cudaEventCreate(&p->ev1))) != CP_OK) break;
        if ((s = cuda_ok(cudaMalloc(&p->cnt, sizeof(unsigned long long) * (C_COUNT + kDepthBins)))) != CP_OK) break;
        p->per_depth = p->cnt + C_COUNT;
        if ((s = cuda_ok(cudaMallocHost(&p->h_cnt, sizeof(unsigned long long) * (C_COUNT + kDepthBins)))) != CP_OK)
            break;
        // single-placement table on 2^16 lambda points over [0.5, 0.99]
        p->tab_n = 1 << 16;
        p->tab_h = (kLambdaMax - kLambdaMin) / (p->tab_n - 1);
        if ((s = cuda_ok(cudaMalloc(&p->tab_t, sizeof(double) * p->tab_n))) != CP_OK) break;
        if ((s = cuda_ok(cudaMalloc(&p->tab_v, sizeof(double) * p->tab_n))) != CP_OK) break;
        k_single_table<<<256, 128, 0, p->stream>>>(kLambdaMin, p->tab_h, p->tab_n, p->tab_t, p->tab_v);
        if ((s = cp_check_launch()) != CP_OK) break;
        if ((s = cuda_ok(cudaStreamSynchronize(p->stream))) != CP_OK) break;
    } while (0);
    if (s != CP_OK) {
        cp_destroy(p);
        return s;
    }
    *out = p;
    return CP_OK;
}

void cp_destroy(cp_prover* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    cp_model_free(p);
    free_graph(p);
    cudaFree(p->d_levels);
    cudaFree(p->d_sched);
    cudaFreeHost(p->h_sched);
    free_levels(p);
    cudaFree(p->cnt);
    cudaFreeHost(p->h_cnt);
    cudaFree(p->tab_t);
    cudaFree(p->tab_v);
    cudaFree(p->slab_single);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
    for (auto& st : p->stage) {
        cudaFree(st.buf);
        if (st.done) cudaEventDestroy(st.done);
    }
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

void* cp_get_stream(cp_prover* p) { return p ? (void*)p->stream : nullptr; }

void cp_request_interrupt(cp_prover* p) {
    if (p) p->interrupt.store(1);
}

void cp_set_chunk_callback(cp_prover* p, cp_chunk_callback cb, void* user) {
    if (!p) return;
    p->chunk_cb = cb;
    p->chunk_user = user;
}

void cp_set_step_callback(cp_prover* p, cp_step_callback cb, void* user) {
    if (!p) return;
    p->step_cb = cb;
    p->step_user = user;
}

cp_status cp_refine(cp_prover* p, const cp_refine_opts* o, cp_refine_report* r) {
    if (!p || !r) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    p->interrupt.store(0);  // a request made while no refinement ran does not stop this one
    return cp_refine_keep_interrupt(p, o, r);
}

// cp_refine without clearing a pending interrupt request (the proof driver's slabs)
__attribute__((visibility("hidden"))) cp_status cp_refine_keep_interrupt(cp_prover* p, const cp_refine_opts* o, cp_refine_report* r) {
    if (!p || !r) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    p->pending = false;
    const double t0 = now_ms();
    std::memset(r, 0, sizeof(*r));
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const int fam = o->family;
    const int D = family_dims(fam);
    LatticeSpec s{fam, {1, 1, 1, 1}, o->seed_lambda[0], o->seed_lambda[1]};
    size_t total = 1;
    for (int d = 0; d < D; ++d) {
        if (o->seed_sizes[d] <= 0) return CP_ERR_INVALID;
        s.n[d] = o->seed_sizes[d];
        total *= (size_t)s.n[d];
    }
    // this call's piece of the lattice: boxes part, part + parts, part + 2 parts, ...
    const size_t parts = o->seed_parts > 1 ? (size_t)o->seed_parts : 1;
    const size_t part = parts > 1 ? (size_t)o->seed_part : 0;
    if (part >= parts) return cp_fail(CP_ERR_INVALID, "cp_refine: seed_part must be in [0, seed_parts)");
    const size_t lattice_total = total;
    total = lattice_total > part ? (lattice_total - part + parts - 1) / parts : 0;
    const size_t cap = o->level_capacity > 0 ? (size_t)o->level_capacity : ((size_t)1 << 25);
    if (total > cap) return CP_ERR_CAPACITY;
    CP_TRY(ensure_levels(p, o->max_depth + 1, D, cap));
    for (auto& L : p->levels) L.n = 0;
    CP_TRY(ensure_slab(p, s.n[0]));
    CP_TRY(cp_launch_slab_single(s, p->slab_single, p->stream));
    k_seed<<<grid_of(k_seed, 128), 128, 0, p->stream>>>(s, p->slab_single, total, part, parts, p->levels[0].b);
    CP_TRY(cp_check_launch());
    p->levels[0].n = total;
    CP_TRY(reset_counters(p));
    return run_refinement(p, *o, r, t0);
}

cp_status cp_proof_defaults(int family, cp_proof_opts* o) {
    if (!o || family < 0 || family > 5) return CP_ERR_INVALID;
    std::memset(o, 0, sizeof(*o));
    o->family = family;
    o->precision = CP_FP64;
    o->engine = CP_ENGINE_GRAPH;
    o->policy = CP_SPLIT_LAMBDA;
    o->max_depth = 24;
    o->slabs = 1;
    o->geometric = 0;
    o->level_capacity = (int64_t)1 << 23;
    // with the coarse seeds below, carrying a parent's lambda-independent terms
    // costs more than it saves (measured on the start proof: 146 against 138 ms)
    o->reuse = 0;
    // the coarsest seed lattice that still proves each family with lambda-only
    // refinement, found by a coordinate-descent search on B200 (each step
    // coarsened one axis while the proof stayed complete with fewer boxes);
    // start and start_end_3d: geometric lambda slabs with a radius lattice per slab (below)
    static const int32_t seeds[6][4] = {{1, 256, 256, 64}, {64, 32, 32, 1},  {64, 64, 64, 16},
                                        {51, 26, 21, 1},   {33, 66, 53, 1},   {41, 17, 17, 4}};
    for (int d = 0; d < 4; ++d) o->seed_sizes[d] = seeds[family][d];
    if (family == CP_START) {
        o->slabs = 18;
        o->geometric = 1;
        o->max_depth = 30;
        o->level_capacity = (int64_t)1 << 24;
        // per slab, the coarsest radius lattice that still proves it, found by a
        // coordinate-descent search on B200 (each step coarsened one radius axis
        // while the slab stayed proved with fewer boxes).  r3 needs no
        // subdivision at all; r1 needs the most, growing toward lambda = 0.99.
        static const int32_t radii[18][3] = {
            {30, 17, 1},   {37, 20, 1},   {41, 27, 1},   {51, 30, 1},   {60, 41, 1},   {67, 57, 1},
            {79, 67, 1},   {93, 71, 1},   {109, 79, 1},  {128, 86, 1},  {144, 96, 1},  {160, 107, 1},
            {176, 118, 1}, {176, 176, 1}, {192, 192, 1}, {208, 177, 1}, {224, 171, 1}, {224, 224, 1}};
        for (int k = 0; k < 18; ++k)
            for (int d = 0; d < 3; ++d) o->slab_radii[k][d] = radii[k][d];
    } else if (family == CP_START_END_3D) {
        // the same geometric slabs, each with its searched radius lattice:
        // 1.30e8 boxes against 2.26e8 for one 64 x 64 x 64 x 16 seed
        o->slabs = 18;
        o->geometric = 1;
        o->seed_sizes[0] = 1;
        static const int32_t radii[18][3] = {
            {26, 41, 8},  {26, 26, 10}, {33, 26, 10}, {33, 33, 10}, {33, 33, 10}, {41, 33, 10},
            {41, 33, 10}, {33, 41, 10}, {41, 41, 10}, {41, 41, 10}, {41, 51, 10}, {41, 51, 10},
            {51, 51, 10}, {51, 51, 10}, {51, 51, 10}, {51, 51, 10}, {51, 51, 10}, {51, 51, 10}};
        for (int k = 0; k < 18; ++k)
            for (int d = 0; d < 3; ++d) o->slab_radii[k][d] = radii[k][d];
    }
    return CP_OK;
}

cp_status cp_prove_family(cp_prover* p, const cp_proof_opts* o, cp_proof_report* r) {
    if (!p || !o || !r || o->family < 0 || o->family > 5 || o->slabs < 1) return CP_ERR_INVALID;
    std::memset(r, 0, sizeof(*r));
    r->first_unresolved_slab = -1;
    const double t0 = now_ms();
    p->interrupt.store(0);
    for (int k = 0; k < o->slabs; ++k) {
        if (p->interrupt.load()) {
            p->interrupt.store(0);
            r->wall_ms = now_ms() - t0;
            return CP_ERR_INTERRUPTED;
        }
        cp_refine_opts ro{};
        ro.family = o->family;
        ro.precision = o->precision;
        ro.policy = o->policy;
        ro.max_depth = o->max_depth;
        for (int d = 0; d < 4; ++d) ro.seed_sizes[d] = o->seed_sizes[d] > 0 ? o->seed_sizes[d] : 1;
        if (k < 32)
            for (int d = 1; d < 4; ++d)
                if (o->slab_radii[k][d - 1] > 0) ro.seed_sizes[d] = o->slab_radii[k][d - 1];
        ro.seed_lambda[0] = proof_slab_cut(*o, k);
        ro.seed_lambda[1] = proof_slab_cut(*o, k + 1);
        ro.level_capacity = o->level_capacity > 0 ? o->level_capacity : ((int64_t)1 << 24);
        ro.engine = o->engine;
        ro.digest = o->digest;
        ro.seed_parts = o->seed_parts;
        ro.seed_part = o->seed_part;
        ro.reuse = o->reuse;
        cp_refine_report rr;
        const cp_status s = cp_refine_keep_interrupt(p, &ro, &rr);
        if (s != CP_OK) {
            r->wall_ms = now_ms() - t0;
            return s;
        }
        r->slabs_done = k + 1;
        r->evaluated += rr.evaluated;
        for (int v = 0; v < 5; ++v) r->verdicts[v] += rr.verdicts[v];
        r->unresolved += rr.unresolved;
        r->clipped += rr.clipped;
        for (int d = 0; d < 64; ++d) r->per_depth[d] += rr.per_depth[d];
        if (rr.max_depth_seen > r->max_depth_seen) r->max_depth_seen = rr.max_depth_seen;
        if (rr.unresolved && r->first_unresolved_slab < 0) r->first_unresolved_slab = k;
        r->device_ms += rr.device_ms;
        r->digest[0] += rr.digest[0];
        r->digest[1] ^= rr.digest[1];
    }
    r->proved = r->unresolved == 0 ? 1 : 0;
    r->wall_ms = now_ms() - t0;
    return CP_OK;
}

cp_status cp_prove_all(cp_prover* p, int precision, int engine, cp_proof_report* reports) {
    if (!p || !reports) return CP_ERR_INVALID;
    for (int f = 0; f < 6; ++f) {
        cp_proof_opts o;
        CP_TRY(cp_proof_defaults(f, &o));
        o.precision = precision;
        o.engine = engine;
        CP_TRY(cp_prove_family(p, &o, &reports[f]));
    }
    return CP_OK;
}

cp_status cp_random_boxes(cp_prover* p, int family, uint64_t seed, int max_label, size_t n, double* lo, double* hi,
                          uint8_t* depth) {
    if (!p || family < 0 || family > 5 || max_label < 0 || max_label > 250 || (n && (!lo || !hi || !depth)))
        return CP_ERR_INVALID;
    if (!n) return CP_OK;
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const BoxList out{lo, hi, depth, n};
    k_random_boxes<<<grid_of(k_random_boxes, 128), 128, 0, p->stream>>>(family, (unsigned long long)seed, max_label, n,
                                                                        table_of(p), out);
    CP_TRY(cp_check_launch());
    return cuda_ok(cudaStreamSynchronize(p->stream));
}

cp_status cp_set_level_variant(cp_prover* p, int family, int precision, int variant) {
    if (!p || family < 0 || family > 5 || precision < 0 || precision > 1 || variant < 0 || variant >= kVariants)
        return CP_ERR_INVALID;
    p->variant[family][precision] = variant;
    return CP_OK;
}

cp_status cp_autotune(cp_prover* p, const cp_refine_opts* o, int* best, double* ms) {
    if (!p || !best) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    const int pr = o->precision ? 1 : 0;
    double best_ms = 1e300;
    int best_v = 0;
    for (int v = 0; v < kVariants; ++v) {
        p->variant[o->family][pr] = v;
        cp_refine_report r;
        CP_TRY(cp_refine(p, o, &r));  // warm-up
        CP_TRY(cp_refine(p, o, &r));
        if (ms) ms[v] = r.device_ms;
        if (r.device_ms < best_ms) {
            best_ms = r.device_ms;
            best_v = v;
        }
    }
    p->variant[o->family][pr] = best_v;
    *best = best_v;
    return CP_OK;
}

cp_status cp_autotune_graph(cp_prover* p, const cp_refine_opts* o, int* block, int* boxes_per_thread, double* ms) {
    if (!p || !block || !boxes_per_thread) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    static const int kBpt[4] = {1, 2, 4, 8};
    cp_refine_opts t = *o;
    t.engine = CP_ENGINE_GRAPH;
    double best_ms = 1e300;
    int best_v = 1, best_b = 2;
    for (int v = 0; v < kGraphVariants; ++v)
        for (int b = 0; b < 4; ++b) {
            t.block = kGraphBlock[v];
            t.boxes_per_thread = kBpt[b];
            cp_refine_report r;
            CP_TRY(cp_refine(p, &t, &r));  // warm-up (also builds the graph)
            CP_TRY(cp_refine(p, &t, &r));
            if (ms) ms[v * 4 + b] = r.device_ms;
            if (r.device_ms < best_ms) {
                best_ms = r.device_ms;
                best_v = v;
                best_b = kBpt[b];
            }
        }
    const int pr = o->precision ? 1 : 0;
    p->graph_variant[o->family][pr] = best_v;
    p->graph_bpt[o->family][pr] = best_b;
    *block = kGraphBlock[best_v];
    *boxes_per_thread = best_b;
    return CP_OK;
}

cp_status cp_refine_boxes(cp_prover* p, const cp_refine_opts* o, const double* lo, const double* hi,
                          const uint8_t* depth, size_t n, cp_refine_report* r) {
    if (!p || !r || (n && (!lo || !hi))) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    p->pending = false;
    p->interrupt.store(0);  // a request made while no refinement ran does not stop this one
    const double t0 = now_ms();
    std::memset(r, 0, sizeof(*r));
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const int D = family_dims(o->family);
    const size_t cap = o->level_capacity > 0 ? (size_t)o->level_capacity : ((size_t)1 << 25);
    if (n > cap) return CP_ERR_CAPACITY;
    CP_TRY(ensure_levels(p, o->max_depth + 1, D, cap));
    for (auto& L : p->levels) L.n = 0;
    if (n) {
        k_copy_seed<<<grid_of(k_copy_seed, 128), 128, 0, p->stream>>>(D, lo, hi, depth, n, p->levels[0].b);
        CP_TRY(cp_check_launch());
    }
    p->levels[0].n = n;
    CP_TRY(reset_counters(p));
    // explicit seeds may carry depths above zero: they stay in level 0's buffer
    // and their children go to level 1; max_depth compares with the box depth
    return run_refinement(p, *o, r, t0);
}

cp_status cp_refine_boxes_host(cp_prover* p, const cp_refine_opts* o, const double* lo, const double* hi,
                               const uint8_t* depth, size_t n, cp_refine_report* r) {
    if (!p || !r || (n && (!lo || !hi))) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    p->pending = false;
    p->interrupt.store(0);  // a request made while no refinement ran does not stop this one
    const double t0 = now_ms();
    std::memset(r, 0, sizeof(*r));
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const int D = family_dims(o->family);
    const size_t cap = o->level_capacity > 0 ? (size_t)o->level_capacity : ((size_t)1 << 25);
    if (n > cap) return CP_ERR_CAPACITY;
    CP_TRY(ensure_levels(p, o->max_depth + 1, D, cap));
    for (auto& L : p->levels) L.n = 0;
    BoxList& b = p->levels[0].b;
    for (int d = 0; d < D && n; ++d) {
        CP_TRY(cuda_ok(cudaMemcpyAsync(b.lo + d * b.cap, lo + d * n, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream)));
        CP_TRY(cuda_ok(cudaMemcpyAsync(b.hi + d * b.cap, hi + d * n, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream)));
    }
    if (n) {
        if (depth)
            CP_TRY(cuda_ok(cudaMemcpyAsync(b.depth, depth, n, cudaMemcpyHostToDevice, p->stream)));
        else
            CP_TRY(cuda_ok(cudaMemsetAsync(b.depth, 0, n, p->stream)));
    }
    p->levels[0].n = n;
    CP_TRY(reset_counters(p));
    return run_refinement(p, *o, r, t0);
}

cp_status cp_stage_boxes_host(cp_prover* p, int slot, const double* lo, const double* hi, const uint8_t* depth,
                              size_t n, int dims) {
    if (!p || slot < 0 || slot > 1 || (dims != 3 && dims != 4) || (n && (!lo || !hi))) return CP_ERR_INVALID;
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    if (!p->copy_stream) CP_TRY(cuda_ok(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking)));
    cp_prover::Stage& st = p->stage[slot];
    if (!st.done) CP_TRY(cuda_ok(cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming)));
    const size_t axis = sizeof(double) * (size_t)dims * n;
    const size_t need = 2 * axis + n;
    if (st.bytes < need) {
        // the slot's previous copy and any refinement reading it have finished
        // (the refinement is synchronous), so the buffer can be replaced
        CP_TRY(cuda_ok(cudaStreamSynchronize(p->copy_stream)));
        cudaFree(st.buf);
        st.buf = nullptr;
        st.bytes = 0;
        CP_TRY(cuda_ok(cudaMalloc(&st.buf, need)));
        st.bytes = need;
    }
    st.n = n;
    st.dims = dims;
    st.has_depth = depth != nullptr;
    if (n) {
        CP_TRY(cuda_ok(cudaMemcpyAsync(st.buf, lo, axis, cudaMemcpyHostToDevice, p->copy_stream)));
        CP_TRY(cuda_ok(cudaMemcpyAsync(st.buf + axis, hi, axis, cudaMemcpyHostToDevice, p->copy_stream)));
        if (depth) CP_TRY(cuda_ok(cudaMemcpyAsync(st.buf + 2 * axis, depth, n, cudaMemcpyHostToDevice, p->copy_stream)));
    }
    CP_TRY(cuda_ok(cudaEventRecord(st.done, p->copy_stream)));
    st.staged = true;
    return CP_OK;
}

cp_status cp_refine_staged(cp_prover* p, const cp_refine_opts* o, int slot, cp_refine_report* r) {
    if (!p || !r || slot < 0 || slot > 1) return CP_ERR_INVALID;
    CP_TRY(check_opts(o));
    cp_prover::Stage& st = p->stage[slot];
    if (!st.staged) return cp_fail(CP_ERR_INVALID, "cp_refine_staged: slot %d holds no staged boxes", slot);
    const int D = family_dims(o->family);
    if (st.dims != D) return cp_fail(CP_ERR_INVALID, "cp_refine_staged: slot %d holds %d-axis boxes", slot, st.dims);
    p->pending = false;
    p->interrupt.store(0);
    const double t0 = now_ms();
    std::memset(r, 0, sizeof(*r));
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const size_t n = st.n;
    const size_t cap = o->level_capacity > 0 ? (size_t)o->level_capacity : ((size_t)1 << 25);
    if (n > cap) return CP_ERR_CAPACITY;
    CP_TRY(ensure_levels(p, o->max_depth + 1, D, cap));
    for (auto& L : p->levels) L.n = 0;
    // the refinement's stream waits for the slot's copy, then moves the boxes
    // into the level stack (device to device)
    CP_TRY(cuda_ok(cudaStreamWaitEvent(p->stream, st.done, 0)));
    // (a kernel, not a device-to-device copy, which could queue on a copy
    // engine behind the next slot's host-to-device copy)
    const double* slo = reinterpret_cast<const double*>(st.buf);
    const double* shi = slo + (size_t)D * n;
    const uint8_t* sdp = st.has_depth ? st.buf + 2 * sizeof(double) * D * n : nullptr;
    if (n) {
        k_copy_seed<<<grid_of(k_copy_seed, 128), 128, 0, p->stream>>>(D, slo, shi, sdp, n, p->levels[0].b);
        CP_TRY(cp_check_launch());
    }
    p->levels[0].n = n;
    CP_TRY(reset_counters(p));
    return run_refinement(p, *o, r, t0);
}

// ------------------------------------------------------------------ resume / checkpoints
cp_status cp_refine_resume(cp_prover* p, cp_refine_report* r) {
    if (!p || !r) return CP_ERR_INVALID;
    if (!p->pending) return cp_fail(CP_ERR_INVALID, "cp_refine_resume: no interrupted refinement in this handle");
    const double t0 = now_ms();
    std::memset(r, 0, sizeof(*r));
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const cp_refine_opts o = p->pending_opts;
    p->pending = false;
    return refine_levels(p, o, r, t0);
}

}  // extern "C"

namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, dims;
    uint32_t opts_size, counter_words;
    uint64_t level_cap;
    uint32_t nlevels, reserved;
    cp_refine_opts opts;
};
constexpr char kCkptMagic[8] = {'C', 'P', 'B', '2', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCkptVersion = 1;
constexpr size_t kCkptStage = (size_t)1 << 22;  // doubles per staging copy

// Copies `count` elements of device array `dev` to `f` through a host buffer.
template <class T>
cp_status dump(std::FILE* f, const T* dev, size_t count, std::vector<unsigned char>& stage, cudaStream_t st) {
    const size_t per = stage.size() / sizeof(T);
    for (size_t off = 0; off < count; off += per) {
        const size_t k = std::min(per, count - off);
        CP_TRY(cuda_ok(cudaMemcpyAsync(stage.data(), dev + off, k * sizeof(T), cudaMemcpyDeviceToHost, st)));
        CP_TRY(cuda_ok(cudaStreamSynchronize(st)));
        if (std::fwrite(stage.data(), sizeof(T), k, f) != k) return cp_fail(CP_ERR_INVALID, "checkpoint: write failed");
    }
    return CP_OK;
}
template <class T>
cp_status load(std::FILE* f, T* dev, size_t count, std::vector<unsigned char>& stage, cudaStream_t st) {
    const size_t per = stage.size() / sizeof(T);
    for (size_t off = 0; off < count; off += per) {
        const size_t k = std::min(per, count - off);
        if (std::fread(stage.data(), sizeof(T), k, f) != k) return cp_fail(CP_ERR_INVALID, "checkpoint: file truncated");
        CP_TRY(cuda_ok(cudaMemcpyAsync(dev + off, stage.data(), k * sizeof(T), cudaMemcpyHostToDevice, st)));
        CP_TRY(cuda_ok(cudaStreamSynchronize(st)));
    }
    return CP_OK;
}
struct FileCloser {
    std::FILE* f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};
}  // namespace

extern "C" {

cp_status cp_checkpoint_save(cp_prover* p, const char* path) {
    if (!p || !path) return CP_ERR_INVALID;
    if (!p->pending) return cp_fail(CP_ERR_INVALID, "cp_checkpoint_save: no interrupted refinement in this handle");
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return cp_fail(CP_ERR_INVALID, "cp_checkpoint_save: cannot open %s", path);
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = kCkptVersion;
    h.dims = (uint32_t)family_dims(p->pending_opts.family);
    h.opts_size = (uint32_t)sizeof(cp_refine_opts);
    h.counter_words = (uint32_t)(C_COUNT + kDepthBins);
    h.level_cap = p->level_cap;
    h.nlevels = (uint32_t)p->levels.size();
    h.opts = p->pending_opts;
    if (std::fwrite(&h, sizeof(h), 1, fc.f) != 1) return cp_fail(CP_ERR_INVALID, "checkpoint: write failed");
    std::vector<uint64_t> n(h.nlevels);
    for (uint32_t l = 0; l < h.nlevels; ++l) n[l] = p->levels[l].n;
    if (std::fwrite(n.data(), sizeof(uint64_t), n.size(), fc.f) != n.size())
        return cp_fail(CP_ERR_INVALID, "checkpoint: write failed");
    std::vector<unsigned char> stage(sizeof(double) * kCkptStage);
    CP_TRY(dump(fc.f, p->cnt, h.counter_words, stage, p->stream));
    for (uint32_t l = 0; l < h.nlevels; ++l) {
        if (!n[l]) continue;
        const BoxList& b = p->levels[l].b;
        for (uint32_t d = 0; d < h.dims; ++d) CP_TRY(dump(fc.f, b.lo + d * b.cap, n[l], stage, p->stream));
        for (uint32_t d = 0; d < h.dims; ++d) CP_TRY(dump(fc.f, b.hi + d * b.cap, n[l], stage, p->stream));
        CP_TRY(dump(fc.f, b.depth, n[l], stage, p->stream));
    }
    if (std::fflush(fc.f) != 0) return cp_fail(CP_ERR_INVALID, "checkpoint: write failed");
    return CP_OK;
}

cp_status cp_checkpoint_load(cp_prover* p, const char* path, cp_refine_opts* opts) {
    if (!p || !path) return CP_ERR_INVALID;
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return cp_fail(CP_ERR_INVALID, "cp_checkpoint_load: cannot open %s", path);
    CkptHeader h;
    if (std::fread(&h, sizeof(h), 1, fc.f) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 ||
        h.version != kCkptVersion || h.opts_size != sizeof(cp_refine_opts) ||
        h.counter_words != (uint32_t)(C_COUNT + kDepthBins))
        return cp_fail(CP_ERR_INVALID, "cp_checkpoint_load: %s is not a checkpoint of this library version", path);
    CP_TRY(check_opts(&h.opts));
    if (h.dims != (uint32_t)family_dims(h.opts.family) || h.nlevels == 0 || h.nlevels > 251 || h.level_cap == 0)
        return cp_fail(CP_ERR_INVALID, "cp_checkpoint_load: inconsistent header in %s", path);
    std::vector<uint64_t> n(h.nlevels);
    if (std::fread(n.data(), sizeof(uint64_t), n.size(), fc.f) != n.size())
        return cp_fail(CP_ERR_INVALID, "checkpoint: file truncated");
    for (uint64_t k : n)
        if (k > h.level_cap) return cp_fail(CP_ERR_INVALID, "cp_checkpoint_load: level larger than its capacity");
    p->pending = false;
    CP_TRY(ensure_levels(p, (int)h.nlevels, (int)h.dims, (size_t)h.level_cap));
    std::vector<unsigned char> stage(sizeof(double) * kCkptStage);
    CP_TRY(load(fc.f, p->cnt, h.counter_words, stage, p->stream));
    for (auto& L : p->levels) L.n = 0;
    for (uint32_t l = 0; l < h.nlevels; ++l) {
        if (!n[l]) continue;
        BoxList& b = p->levels[l].b;
        for (uint32_t d = 0; d < h.dims; ++d) CP_TRY(load(fc.f, b.lo + d * b.cap, n[l], stage, p->stream));
        for (uint32_t d = 0; d < h.dims; ++d) CP_TRY(load(fc.f, b.hi + d * b.cap, n[l], stage, p->stream));
        CP_TRY(load(fc.f, b.depth, n[l], stage, p->stream));
        // a checkpoint carries no lambda-independent terms: the loaded boxes recompute them
        if (p->levels[l].aux)
            CP_TRY(cuda_ok(cudaMemsetAsync(p->levels[l].aux + 3 * b.cap, 0, sizeof(double) * n[l], p->stream)));
        p->levels[l].n = (size_t)n[l];
    }
    p->pending = true;
    p->pending_opts = h.opts;
    if (opts) *opts = h.opts;
    return CP_OK;
}

cp_status cp_reference_step(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                            double* first_critical, double* err_box) {
    if (!p || family < 0 || family > 5 || !first_critical) return CP_ERR_INVALID;
    p->pending = false;  // the counters are reused
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const int D = family_dims(family);
    LatticeSpec s{family, {1, 1, 1, 1}, la_lb, la_ub};
    int rs[4];
    reference_sizes(family, rs);
    for (int d = 0; d < D; ++d) {
        s.n[d] = sizes ? sizes[d] : rs[d];
        if (s.n[d] <= 0) return CP_ERR_INVALID;
    }
    CP_TRY(ensure_slab(p, s.n[0]));
    CP_TRY(cp_launch_slab_single(s, p->slab_single, p->stream));
    CP_TRY(reset_counters(p));
    const unsigned long long none = (unsigned long long)s.n[0], no_bits = ~0ull;
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->cnt + C_BEST_SLAB, &none, sizeof(none), cudaMemcpyHostToDevice, p->stream)));
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->cnt + C_NOFIT_SLAB, &none, sizeof(none), cudaMemcpyHostToDevice, p->stream)));
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->cnt + C_TRAP_SLAB, &none, sizeof(none), cudaMemcpyHostToDevice, p->stream)));
    CP_TRY(cuda_ok(cudaMemcpyAsync(p->cnt + C_FIRST_BITS, &no_bits, sizeof(no_bits), cudaMemcpyHostToDevice, p->stream)));
    CP_TRY(cuda_ok(cudaStreamSynchronize(p->stream)));
    size_t per_slab = 1;
    for (int d = 1; d < D; ++d) per_slab *= (size_t)s.n[d];
    const size_t wave_boxes = (size_t)1 << 23;
    const int wave_slabs = (int)std::max<size_t>(1, wave_boxes / per_slab);
    RefKernel k = ref_kernel(family);
    const unsigned grid = grid_of(k, kEvalBlock);
    for (int s0 = 0; s0 < s.n[0]; s0 += wave_slabs) {
        const int ns = std::min(wave_slabs, s.n[0] - s0);
        RefArgs a{s, p->slab_single, s0, (size_t)ns * per_slab, p->cnt, 0, nullptr, nullptr, 0};
        k<<<grid, kEvalBlock, 0, p->stream>>>(a);
        CP_TRY(cp_check_launch());
        CP_TRY(read_counters(p));
        const unsigned long long stop = (unsigned long long)(s0 + ns - 1);
        if (p->h_cnt[C_BEST_SLAB] < (unsigned long long)s.n[0] || p->h_cnt[C_TRAP_SLAB] <= stop ||
            p->h_cnt[C_NOFIT_SLAB] <= stop)
            break;
    }
    // Every box of the slabs up to the first failing slab was evaluated.  The
    // reference kernel visits each thread's boxes lambda slab by lambda slab and
    // returns at the thread's first failing box, so it certainly reaches (and
    // traps on) a box of a slab below the first failing slab, or of any slab when
    // no box fails; in the first failing slab itself that depends on its thread
    // order, and later slabs are not evaluated here.  The certain cases are errors.
    const unsigned long long best = p->h_cnt[C_BEST_SLAB];  // == n[0] when no box fails
    const bool trap_hit = p->h_cnt[C_TRAP_SLAB] < best, nofit_hit = p->h_cnt[C_NOFIT_SLAB] < best;
    if (err_box && (trap_hit || nofit_hit) && p->h_cnt[C_ERRBOX_CLAIM]) {
        for (int j = 0; j < 8; ++j) {
            unsigned long long b = p->h_cnt[C_ERRBOX + j];
            std::memcpy(&err_box[j], &b, 8);
        }
    }
    if (trap_hit) return CP_ERR_TRAP_SITE;
    if (nofit_hit) return CP_ERR_NOFIT;
    *first_critical = p->h_cnt[C_FIRST_BITS] == ~0ull ? INFINITY : ordered_value(p->h_cnt[C_FIRST_BITS]);
    return CP_OK;
}

cp_status cp_prove_family_reference(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                                    int64_t max_launches, double* trace, cp_reference_report* r) {
    if (!p || !r || family < 0 || family > 5) return CP_ERR_INVALID;
    p->pending = false;  // the counters are reused
    std::memset(r, 0, sizeof(*r));
    const double t0 = now_ms();
    struct Lb {
        bool operator()(const std::pair<double, double>& a, const std::pair<double, double>& b) const {
            return a.first > b.first;
        }
    };
    std::priority_queue<std::pair<double, double>, std::vector<std::pair<double, double>>, Lb> q;
    q.push({la_lb, la_ub});
    p->interrupt.store(0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cp_status status = CP_OK;
    while (!q.empty()) {
        if (max_launches > 0 && r->launches >= max_launches) {
            status = CP_ERR_NOT_PROVED;
            break;
        }
        const auto cur = q.top();
        q.pop();
        if (p->step_cb) p->step_cb(p->step_user, cur.first, cur.second);
        double first = INFINITY;
        cudaEventRecord(e0, p->stream);
        cp_status s = cp_reference_step(p, family, cur.first, cur.second, sizes, &first, nullptr);
        cudaEventRecord(e1, p->stream);
        cudaEventSynchronize(e1);
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        r->device_ms += t;
        r->boxes_evaluated += (int64_t)p->h_cnt[C_EVALUATED];
        if (trace) {
            trace[3 * r->launches + 0] = cur.first;
            trace[3 * r->launches + 1] = cur.second;
            trace[3 * r->launches + 2] = first;
        }
        r->launches++;
        if (s != CP_OK) {
            r->remaining[0] = cur.first;
            r->remaining[1] = cur.second;
            status = s;
            break;
        }
        if (p->interrupt.load()) {
            p->interrupt.store(0);
            r->interrupted = 1;
            if (first != INFINITY) {
                r->remaining[0] = cur.first, r->remaining[1] = cur.second;
            } else if (!q.empty()) {
                r->remaining[0] = q.top().first, r->remaining[1] = q.top().second;
            } else {
                r->proved = 1;
                break;
            }
            status = CP_ERR_INTERRUPTED;
            break;
        }
        // run_kernel.cuh:110-127
        if (first != INFINITY) {
            const double width_before = cur.second - cur.first;
            const double width_after = cur.second - first;
            if (width_before >= 2 * width_after) {
                q.push({first, cur.second});
            } else {
                const double mid = 0.5 * (first + cur.second);
                if (first < mid) q.push({first, mid});
                if (mid <= cur.second) q.push({mid, cur.second});
            }
        }
    }
    if (status == CP_OK) r->proved = 1;
    if (status == CP_ERR_NOT_PROVED && !q.empty()) {
        r->remaining[0] = q.top().first;
        r->remaining[1] = q.top().second;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    r->wall_ms = now_ms() - t0;
    return status;
}

cp_status cp_reference_criticals(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                                 size_t max_boxes, double* boxes, uint8_t* handles, size_t* count) {
    if (!p || family < 0 || family > 5 || !count || (max_boxes && (!boxes || !handles))) return CP_ERR_INVALID;
    p->pending = false;  // the counters are reused
    CP_TRY(cuda_ok(cudaSetDevice(p->device)));
    const int D = family_dims(family);
    LatticeSpec s{family, {1, 1, 1, 1}, la_lb, la_ub};
    int rs[4];
    reference_sizes(family, rs);
    for (int d = 0; d < D; ++d) {
        s.n[d] = sizes ? sizes[d] : rs[d];
        if (s.n[d] <= 0) return CP_ERR_INVALID;
    }
    CP_TRY(ensure_slab(p, s.n[0]));
    CP_TRY(cp_launch_slab_single(s, p->slab_single, p->stream));
    CP_TRY(reset_counters(p));
    double* dboxes = nullptr;
    uint8_t* dh = nullptr;
    const size_t cap = max_boxes ? max_boxes : 1;
    CP_TRY(cuda_ok(cudaMalloc(&dboxes, sizeof(double) * 8 * cap)));
    if (cuda_ok(cudaMalloc(&dh, cap)) != CP_OK) {
        cudaFree(dboxes);
        return CP_ERR_NOMEM;
    }
    size_t per_slab = 1;
    for (int d = 1; d < D; ++d) per_slab *= (size_t)s.n[d];
    RefKernel k = ref_kernel(family);
    RefArgs a{s, p->slab_single, 0, (size_t)s.n[0] * per_slab, p->cnt, 1, dboxes, dh, max_boxes};
    k<<<grid_of(k, kEvalBlock), kEvalBlock, 0, p->stream>>>(a);
    cp_status st = cp_check_launch();
    if (st == CP_OK) st = read_counters(p);
    if (st == CP_OK) {
        *count = (size_t)p->h_cnt[C_COLLECT];
        const size_t m = std::min(*count, max_boxes);
        if (m) {
            st = cuda_ok(cudaMemcpy(boxes, dboxes, sizeof(double) * 8 * m, cudaMemcpyDeviceToHost));
            if (st == CP_OK) st = cuda_ok(cudaMemcpy(handles, dh, m, cudaMemcpyDeviceToHost));
        }
    }
    cudaFree(dboxes);
    cudaFree(dh);
    return st;
}

}  // extern "C"
