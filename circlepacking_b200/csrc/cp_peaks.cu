// Peak-throughput probes of the FP64 primitives (the roofline denominators of
// the compute-bound criterion kernels).  Each kernel runs 8 independent chains
// per thread at full occupancy; the chains' results are stored so that no work
// is dead code.
#include <cuda_runtime.h>

#include "cp_common.h"
#include "cp_fp64.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 256;

template <int OP>
__global__ void __launch_bounds__(256) k_probe(double seed, double* out) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = seed + 1e-3 * (threadIdx.x + c);
    const double a = 0.999999, b = 1e-9;
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            if (OP == 0) x[c] = __fma_rn(x[c], a, b);
            if (OP == 1) x[c] = __dadd_rd(x[c], b);
            if (OP == 2) x[c] = __dmul_rd(x[c], a);
            if (OP == 3) x[c] = __ddiv_rd(x[c], 1.0000001);
            if (OP == 4) x[c] = asin(x[c]) * 0.5 + 0.25;
            if (OP == 5) x[c] = cpb::div_rd(x[c], 1.0000001);
            if (OP == 6) x[c] = cpb::div_dir<false, 1>(x[c], 1.0000001);
            if (OP == 7) x[c] = cpb::div_dir<false, 0>(x[c], 1.0000001);
        }
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_probe_ffma(float seed, float* out) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = seed + 1e-3f * (threadIdx.x + c);
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = __fmaf_rn(x[c], 0.9999f, 1e-7f);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class K, class A>
double rate_of(K k, A seed, void* out, int grid, int block, int reps) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k<<<grid, block>>>(seed, (decltype(seed)*)out);
    cudaEventRecord(e0);
    for (int r = 0; r < reps; ++r) k<<<grid, block>>>(seed, (decltype(seed)*)out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double ops = (double)grid * block * kChains * kIters * reps;
    return ops / (ms * 1e-3);
}

}  // namespace

extern "C" cp_status cp_measure_primitives(int device, double* rates) {
    if (!rates) return CP_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return cp_record_cuda_error(cudaGetLastError(), CP_ERR_NO_DEVICE);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int block = 256, grid = sms * 8;
    void* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * grid * block) != cudaSuccess)
        return cp_record_cuda_error(cudaGetLastError(), CP_ERR_NOMEM);
    rates[0] = rate_of(k_probe<0>, 0.5, out, grid, block, 20);
    rates[1] = rate_of(k_probe<1>, 0.5, out, grid, block, 20);
    rates[2] = rate_of(k_probe<2>, 0.5, out, grid, block, 20);
    rates[3] = rate_of(k_probe<3>, 0.5, out, grid, block, 4);
    rates[4] = rate_of(k_probe<4>, 0.5, out, grid, block, 4);
    rates[5] = rate_of(k_probe_ffma, 0.5f, out, grid, block, 20);
    rates[6] = rate_of(k_probe<5>, 0.5, out, grid, block, 4);
    rates[7] = rate_of(k_probe<6>, 0.5, out, grid, block, 4);
    rates[8] = rate_of(k_probe<7>, 0.5, out, grid, block, 4);
    cudaFree(out);
    return cp_check_launch();
}
