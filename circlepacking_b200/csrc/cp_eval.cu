// Stateless device entry points: per-box evaluation, lattice generation,
// single-placement bounds and the diagnostics primitives.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "cp_common.h"
#include "cp_families.cuh"
#include "cp_fp32.cuh"
#include "cp_lattice.cuh"

using namespace cpb;

namespace {

// ------------------------------------------------------------------ kernels
template <int FAM, int MODE>
__global__ void __launch_bounds__(kEvalBlock) k_eval_fp64(const double* __restrict__ lo, const double* __restrict__ hi,
                                                          size_t n, size_t stride, uint8_t* __restrict__ verdict,
                                                          uint8_t* __restrict__ mask, const uint8_t* __restrict__ order,
                                                          double* __restrict__ trace) {
    constexpr int D = family_dims(FAM);
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        double l[4], h[4];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            l[d] = __ldg(lo + d * stride + i);
            h[d] = __ldg(hi + d * stride + i);
        }
        const int ord = order ? order[i] : 0;
        Verdict v = eval_box<FAM, MODE>(l, h, ord, trace ? trace + 16 * i : nullptr);
        verdict[i] = v.verdict;
        mask[i] = v.mask;
    }
}

// FP32 enclosure pass; boxes it cannot prove are re-evaluated in FP64 by the
// same thread (decide mode: the FP64 result; full mode: the full FP64 mask).
template <int FAM, int MODE>
__global__ void __launch_bounds__(kEvalBlock) k_eval_prefilter(const double* __restrict__ lo,
                                                               const double* __restrict__ hi, size_t n, size_t stride,
                                                               uint8_t* __restrict__ verdict, uint8_t* __restrict__ mask,
                                                               const uint8_t* __restrict__ order,
                                                               double* __restrict__ trace) {
    constexpr int D = family_dims(FAM);
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        double l[4], h[4];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            l[d] = __ldg(lo + d * stride + i);
            h[d] = __ldg(hi + d * stride + i);
        }
        const int ord = order ? order[i] : 0;
        uint8_t pmask = 0;
        const int pre = prefilter_box<FAM>(l, h, ord, MODE == FULL, &pmask);
        Verdict v;
        if (pre == PF_UNDECIDED)
            v = eval_box<FAM, MODE>(l, h, ord, trace ? trace + 16 * i : nullptr);
        else
            v = {pre == PF_PROVED ? V_PROVED : pre == PF_EMPTY ? V_EMPTY : pre == PF_NOFIT ? V_NOFIT : V_CRITICAL,
                 pmask};
        verdict[i] = v.verdict;
        mask[i] = v.mask;
    }
}

// The FP32 pre-pass's directed division against the CUDA intrinsics it replaces.
__global__ void k_fdiv_check(const float* __restrict__ a, const float* __restrict__ b, size_t n,
                             float* __restrict__ out) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        out[4 * i + 0] = f32::fdiv_rd(a[i], b[i]);
        out[4 * i + 1] = f32::fdiv_ru(a[i], b[i]);
        out[4 * i + 2] = __fdiv_rd(a[i], b[i]);
        out[4 * i + 3] = __fdiv_ru(a[i], b[i]);
    }
}

// The library's directed division against the CUDA intrinsics it replaces.
__global__ void k_div_check(const double* __restrict__ a, const double* __restrict__ b, size_t n,
                            double* __restrict__ out) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        out[4 * i + 0] = div_rd(a[i], b[i]);
        out[4 * i + 1] = div_ru(a[i], b[i]);
        out[4 * i + 2] = __ddiv_rd(a[i], b[i]);
        out[4 * i + 3] = __ddiv_ru(a[i], b[i]);
    }
}

__global__ void k_single_placement(const double* __restrict__ lam, size_t n, double* __restrict__ out) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) out[i] = single_placement(lam[i]);
}

// single placement bound of each lambda slab's lower end
__global__ void k_slab_single(LatticeSpec s, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n[0]; i += gridDim.x * blockDim.x)
        out[i] = single_placement(subinterval(Iv{s.outer_lo, s.outer_hi}, i, s.n[0]).lo);
}

__global__ void k_lattice(LatticeSpec s, const double* __restrict__ slab_single, const int64_t* __restrict__ index,
                          size_t n, double* __restrict__ lo, double* __restrict__ hi, size_t stride,
                          uint8_t* __restrict__ visited) {
    const int D = family_dims(s.fam);
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += step) {
        int64_t rem = index[t];
        int ix[4] = {0, 0, 0, 0};
        for (int d = D - 1; d >= 0; --d) {
            ix[d] = (int)(rem % s.n[d]);
            rem /= s.n[d];
        }
        double l[4], h[4];
        const bool v = lattice_box(s, ix, slab_single[ix[0]], l, h);
        for (int d = 0; d < D; ++d) {
            lo[d * stride + t] = l[d];
            hi[d * stride + t] = h[d];
        }
        if (visited) visited[t] = v ? 1 : 0;
    }
}

__global__ void k_primitive(int kind, const double* __restrict__ a, size_t n, double* __restrict__ out,
                            uint8_t* __restrict__ trap) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        Iv a0{a[i], a[n + i]}, a1{a[2 * n + i], a[3 * n + i]}, a2{a[4 * n + i], a[5 * n + i]};
        bool t = false;
        Iv r{0.0, 0.0};
        switch (kind) {
        case 0: r = ca_inner_inner(a0, a1, a2, t); break;
        case 1: r = ca_outer_inner(a0, a1, a2, t); break;
        case 2: r = ca_inner_outer(a0, a1, a2, t); break;
        case 3: r = ca_outer_outer(a0, a1, t); break;
        case 4: r = {semi_outer_lo(a0), semi_outer_hi(a0)}; break;
        case 5: r = {semi_inner_lo(a0, a1), semi_inner_hi(a0, a1)}; break;
        }
        out[i] = r.lo;
        out[n + i] = r.hi;
        if (trap) trap[i] = t ? 1 : 0;
    }
}

__global__ void k_asin_pad(const double* __restrict__ x, size_t n, double* __restrict__ rd, double* __restrict__ ru) {
    const size_t step = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        rd[i] = asin_rd(x[i]);
        ru[i] = asin_ru(x[i]);
    }
}

template <class K>
unsigned grid_for(K kernel, size_t n, int block) {
    static thread_local int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    size_t want = (n + block - 1) / block;
    size_t cap = (size_t)sms * (size_t)per_sm;
    size_t g = want < cap ? want : cap;
    return (unsigned)(g ? g : 1);
}

template <int FAM, int MODE>
cp_status launch_eval(int precision, const double* lo, const double* hi, size_t n, size_t stride, uint8_t* verdict,
                      uint8_t* mask, const uint8_t* order, double* trace, cudaStream_t st) {
    if (precision == CP_FP64) {
        auto k = k_eval_fp64<FAM, MODE>;
        k<<<grid_for(k, n, kEvalBlock), kEvalBlock, 0, st>>>(lo, hi, n, stride, verdict, mask, order, trace);
    } else {
        auto k = k_eval_prefilter<FAM, MODE>;
        k<<<grid_for(k, n, kEvalBlock), kEvalBlock, 0, st>>>(lo, hi, n, stride, verdict, mask, order, trace);
    }
    return cp_check_launch();
}

template <int FAM>
cp_status launch_eval_mode(int precision, int mode, const double* lo, const double* hi, size_t n, size_t stride,
                           uint8_t* verdict, uint8_t* mask, const uint8_t* order, double* trace, cudaStream_t st) {
    if (mode == CP_EVAL_FULL) return launch_eval<FAM, FULL>(precision, lo, hi, n, stride, verdict, mask, order, trace, st);
    return launch_eval<FAM, DECIDE>(precision, lo, hi, n, stride, verdict, mask, order, nullptr, st);
}

std::mutex g_host_mu;
struct HostScratch {
    void* p = nullptr;
    size_t bytes = 0;
} g_host_scratch;

}  // namespace

// ------------------------------------------------------------------ internal API
cp_status cp_launch_eval(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                         size_t stride, uint8_t* verdict, uint8_t* mask, const uint8_t* order, double* trace,
                         cudaStream_t st) {
    switch (family) {
    case F_START: return launch_eval_mode<F_START>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    case F_START_END_2D:
        return launch_eval_mode<F_START_END_2D>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    case F_START_END_3D:
        return launch_eval_mode<F_START_END_3D>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    case F_MIDDLE: return launch_eval_mode<F_MIDDLE>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    case F_END_2D: return launch_eval_mode<F_END_2D>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    case F_END_3D: return launch_eval_mode<F_END_3D>(precision, mode, lo, hi, n, stride, verdict, mask, order, trace, st);
    }
    return CP_ERR_INVALID;
}

cp_status cp_launch_slab_single(const LatticeSpec& s, double* out, cudaStream_t st) {
    const int block = 64;
    k_slab_single<<<(s.n[0] + block - 1) / block, block, 0, st>>>(s, out);
    return cp_check_launch();
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int cp_family_dims(int family) {
    if (family < 0 || family > 5) return -1;
    return family_dims(family);
}

int cp_family_criteria(int family) {
    static const int k[6] = {2, 1, 1, 4, 2, 2};
    if (family < 0 || family > 5) return -1;
    return k[family];
}

cp_status cp_eval_boxes(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                        size_t stride, uint8_t* verdict, uint8_t* mask, const uint8_t* order, double* trace,
                        void* stream) {
    if (family < 0 || family > 5 || (precision != CP_FP64 && precision != CP_FP32_PREFILTER) ||
        (mode != CP_EVAL_FULL && mode != CP_EVAL_DECIDE) || stride < n)
        return CP_ERR_INVALID;
    if (n == 0) return CP_OK;
    if (!lo || !hi || !verdict || !mask) return CP_ERR_INVALID;
    return cp_launch_eval(family, precision, mode, lo, hi, n, stride, verdict, mask, order, trace,
                          (cudaStream_t)stream);
}

cp_status cp_eval_boxes_host(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                             uint8_t* verdict, uint8_t* mask) {
    if (family < 0 || family > 5) return CP_ERR_INVALID;
    if (n == 0) return CP_OK;
    if (!lo || !hi || !verdict || !mask) return CP_ERR_INVALID;
    const int D = family_dims(family);
    const size_t box_bytes = sizeof(double) * (size_t)D * n;
    const size_t need = 2 * box_bytes + 2 * n;
    std::lock_guard<std::mutex> lock(g_host_mu);
    if (g_host_scratch.bytes < need) {
        if (g_host_scratch.p) cudaFree(g_host_scratch.p);
        g_host_scratch.p = nullptr;
        g_host_scratch.bytes = 0;
        if (cudaMalloc(&g_host_scratch.p, need) != cudaSuccess) return cp_record_cuda_error(cudaGetLastError(), CP_ERR_NOMEM);
        g_host_scratch.bytes = need;
    }
    char* base = (char*)g_host_scratch.p;
    double* dlo = (double*)base;
    double* dhi = (double*)(base + box_bytes);
    uint8_t* dv = (uint8_t*)(base + 2 * box_bytes);
    uint8_t* dm = dv + n;
    cudaError_t e;
    if ((e = cudaMemcpy(dlo, lo, box_bytes, cudaMemcpyHostToDevice)) != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    if ((e = cudaMemcpy(dhi, hi, box_bytes, cudaMemcpyHostToDevice)) != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    cp_status s = cp_launch_eval(family, precision, mode, dlo, dhi, n, n, dv, dm, nullptr, nullptr, 0);
    if (s != CP_OK) return s;
    if ((e = cudaMemcpy(verdict, dv, n, cudaMemcpyDeviceToHost)) != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    if ((e = cudaMemcpy(mask, dm, n, cudaMemcpyDeviceToHost)) != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    return CP_OK;
}

cp_status cp_lattice_boxes(int family, double outer_lb, double outer_ub, const int32_t* sizes, const int64_t* index,
                           size_t n, double* lo, double* hi, size_t stride, uint8_t* visited, void* stream) {
    if (family < 0 || family > 5 || !sizes || stride < n) return CP_ERR_INVALID;
    const int D = family_dims(family);
    LatticeSpec s{family, {1, 1, 1, 1}, outer_lb, outer_ub};
    for (int d = 0; d < D; ++d) {
        if (sizes[d] <= 0) return CP_ERR_INVALID;
        s.n[d] = sizes[d];
    }
    if (n == 0) return CP_OK;
    if (!index || !lo || !hi) return CP_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    double* slab = nullptr;
    cudaError_t e = cudaMallocAsync(&slab, sizeof(double) * (size_t)s.n[0], st);
    if (e != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_NOMEM);
    cp_status rc = cp_launch_slab_single(s, slab, st);
    if (rc == CP_OK) {
        k_lattice<<<grid_for(k_lattice, n, 128), 128, 0, st>>>(s, slab, index, n, lo, hi, stride, visited);
        rc = cp_check_launch();
    }
    cudaFreeAsync(slab, st);
    return rc;
}

cp_status cp_single_placement(const double* lb_lambda, size_t n, double* out, void* stream) {
    if (n == 0) return CP_OK;
    if (!lb_lambda || !out) return CP_ERR_INVALID;
    k_single_placement<<<grid_for(k_single_placement, n, 128), 128, 0, (cudaStream_t)stream>>>(lb_lambda, n, out);
    return cp_check_launch();
}

cp_status cp_eval_primitive(int kind, const double* args, size_t n, double* out, uint8_t* trap, void* stream) {
    if (kind < 0 || kind > 5) return CP_ERR_INVALID;
    if (n == 0) return CP_OK;
    if (!args || !out) return CP_ERR_INVALID;
    k_primitive<<<grid_for(k_primitive, n, 128), 128, 0, (cudaStream_t)stream>>>(kind, args, n, out, trap);
    return cp_check_launch();
}

cp_status cp_asin_pad(const double* x, size_t n, double* rd, double* ru, void* stream) {
    if (n == 0) return CP_OK;
    if (!x || !rd || !ru) return CP_ERR_INVALID;
    k_asin_pad<<<grid_for(k_asin_pad, n, 128), 128, 0, (cudaStream_t)stream>>>(x, n, rd, ru);
    return cp_check_launch();
}

cp_status cp_div_check(const double* a, const double* b, size_t n, double* out, void* stream) {
    if (n == 0) return CP_OK;
    if (!a || !b || !out) return CP_ERR_INVALID;
    k_div_check<<<grid_for(k_div_check, n, 128), 128, 0, (cudaStream_t)stream>>>(a, b, n, out);
    return cp_check_launch();
}

cp_status cp_fdiv_check(const float* a, const float* b, size_t n, float* out, void* stream) {
    if (n == 0) return CP_OK;
    if (!a || !b || !out) return CP_ERR_INVALID;
    k_fdiv_check<<<grid_for(k_fdiv_check, n, 128), 128, 0, (cudaStream_t)stream>>>(a, b, n, out);
    return cp_check_launch();
}

}  // extern "C"
