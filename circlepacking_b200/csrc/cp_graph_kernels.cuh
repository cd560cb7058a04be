// Kernels of the device-driven refinement loop (cp_graph.cu): the scheduler
// and the persistent level kernel.  Instantiated per precision in
// cp_graph_fp64.cu / cp_graph_fp32.cu so the two compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "cp_level.cuh"

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

}  // namespace cpb
