// Kernels of the device-driven refinement loop (cp_graph.cu): the scheduler
// and the persistent level kernel.  Instantiated per precision in
// cp_graph_fp64.cu / cp_graph_fp32.cu so the two compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "cp_level.cuh"
#include "cp_tc.cuh"

namespace cpb {

// Block-size variants of the persistent kernel and their register caps
// (BLOCK * REGS <= 65536 so at least one block fits an SM).
constexpr int kGraphVariants = 5;
constexpr int kGraphBlock[kGraphVariants] = {64, 128, 256, 512, 1024};
__host__ __device__ constexpr int graph_regs(int block) { return block >= 1024 ? 64 : 96; }

struct PersistArgs {
    const BoxList* levels;  // device array [nlevels]
    DevSched* sched;
    unsigned long long* cnt;
    unsigned long long* per_depth;
    SingleTable tab;
    int policy, max_depth, bpt;
    double lambda_scale;
    const uint8_t* axis_hint;   // per box of the job, indexed from job.begin
    const uint8_t* order_hint;
    int digest;
};

// The chunk of the current job: warps claim 32 * bpt consecutive boxes at a
// time from sched->claim until the job is exhausted, so blocks that meet cheap
// boxes (early exits, proved or empty boxes) take more of the work.
template <int FAM, int PREC, int BLOCK>
__global__ void __launch_bounds__(BLOCK) __maxnreg__(graph_regs(BLOCK)) k_level_persist(PersistArgs pa) {
    __shared__ LevelSmem<BLOCK / 32> sm;
    const DevJob job = pa.sched->job;
    if (job.count == 0) return;  // uniform over the grid
    LevelArgs a;
    a.in = pa.levels[job.in_level];
    a.begin = job.begin;
    a.count = job.count;
    a.out = job.out_level >= 0 ? pa.levels[job.out_level] : BoxList{nullptr, nullptr, nullptr, 0};
    a.cnt = pa.cnt;
    a.per_depth = pa.per_depth;
    a.tab = pa.tab;
    a.policy = pa.policy;
    a.lambda_scale = pa.lambda_scale;
    a.max_depth = job.out_level >= 0 ? pa.max_depth : 0;
    a.axis_hint = pa.axis_hint;
    a.order_hint = pa.order_hint;
    a.digest = pa.digest;
    level_smem_init(sm);
    __syncthreads();
    unsigned handles = 0;
    const int lane = threadIdx.x & 31;
    const unsigned long long per = 32ull * (unsigned long long)pa.bpt;
    for (;;) {
        unsigned long long start = 0;
        if (lane == 0) start = atomicAdd(&pa.sched->claim, per);
        start = __shfl_sync(0xffffffffu, start, 0);
        if (start >= job.count) break;
        for (int b = 0; b < pa.bpt; ++b) {
            const unsigned long long j0 = start + 32ull * (unsigned long long)b;
            if (j0 >= job.count) break;
            level_step<FAM, PREC>(a, (size_t)(j0 + (unsigned long long)lane), sm, handles);
        }
    }
    level_flush(a, sm, handles);
}

// The persistent level kernel with the proposal network run inline: a CTA of
// 128 threads claims 128 boxes of the job at a time, computes their features,
// runs the network's forward pass on the tensor cores (tcgen05, accumulators in
// 64 tensor-memory columns, tc::net_forward), and each thread evaluates its box
// with the criterion order and split axis the network proposes.  The verdicts
// are the interval kernels' own; a timed-out tensor-core wait raises E_TC.
struct NetArgs {
    const tc::bf16* views;
    const float* master;
    int wait_limit;
    int want_order, want_axis;
};
constexpr int kNetBlock = tc::kTcRows;  // one box per thread of a 128-thread CTA
constexpr int kNetMaxCtasPerSm = 512 / (int)tc::kNetCols;  // tensor memory: 512 columns per SM

// (__launch_bounds__ with 5 resident CTAs caps the registers near the 96 of the
// plain persistent kernel's 128-thread shape)
template <int FAM, int PREC>
__global__ void __launch_bounds__(kNetBlock, 5) k_level_persist_net(PersistArgs pa, NetArgs na) {
    constexpr int D = family_dims(FAM);
    __shared__ LevelSmem<kNetBlock / 32> sm;
    __shared__ __align__(128) tc::NetSmem net;
    __shared__ unsigned long long claim;
    const DevJob job = pa.sched->job;
    if (job.count == 0) return;  // uniform over the grid
    LevelArgs a;
    a.in = pa.levels[job.in_level];
    a.begin = job.begin;
    a.count = job.count;
    a.out = job.out_level >= 0 ? pa.levels[job.out_level] : BoxList{nullptr, nullptr, nullptr, 0};
    a.cnt = pa.cnt;
    a.per_depth = pa.per_depth;
    a.tab = pa.tab;
    a.policy = pa.policy;
    a.lambda_scale = pa.lambda_scale;
    a.max_depth = job.out_level >= 0 ? pa.max_depth : 0;
    a.axis_hint = nullptr;
    a.order_hint = nullptr;
    a.digest = pa.digest;
    level_smem_init(sm);
    tc::net_setup(net, na.views, na.master);
    __syncthreads();
    unsigned handles = 0;
    bool ok = true;
    for (;;) {
        if (threadIdx.x == 0) claim = atomicAdd(&pa.sched->claim, (unsigned long long)kNetBlock);
        __syncthreads();
        const unsigned long long start = claim;
        __syncthreads();  // every thread has read the claim before it is replaced
        if (start >= job.count) break;  // uniform over the CTA
        const size_t j = (size_t)(start + threadIdx.x);
        float f[tc::NK];
        if (j < job.count) {
            const size_t i = a.begin + j;
            double lo[4], hi[4];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                lo[d] = a.in.lo[d * a.in.cap + i];
                hi[d] = a.in.hi[d * a.in.cap + i];
            }
            const int dep = a.in.depth[i];
            tc::box_features_fast<D>(lo, hi, dep == 0xFF ? 0 : dep, f);
        } else {
#pragma unroll
            for (int k = 0; k < tc::NK; ++k) f[k] = 0.f;
        }
        float z[tc::NO];
        if (!(ok = tc::net_forward(net, f, z, na.wait_limit))) break;
        int ord = -1, ax = -1;
        if (na.want_order) {
            if (FAM == F_MIDDLE)
                ord = fmaxf(z[2], z[3]) > fmaxf(z[0], z[1]) ? 1 : 0;
            else if (FAM == F_END_2D || FAM == F_END_3D)
                ord = z[1] > z[0] ? 1 : 0;
            else
                ord = 0;
        }
        if (na.want_axis) {
            ax = 0;
            float best = z[4];
#pragma unroll
            for (int d = 1; d < D; ++d)
                if (z[4 + d] > best) {
                    best = z[4 + d];
                    ax = d;
                }
        }
        level_step<FAM, PREC>(a, j, sm, handles, ord, ax);
    }
    if (!ok && threadIdx.x == 0) atomicOr(&a.cnt[C_ERR], (unsigned long long)E_TC);
    tc::net_teardown(net, ok);
    level_flush(a, sm, handles);
}

}  // namespace cpb
