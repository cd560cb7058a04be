// TEST INFRASTRUCTURE ONLY -- shared helpers of the reference-derived GPU checker.
//
// Each ref_<file>.cu translation unit #includes one of the reference's
// lane_packing/*_configuration.cu files unchanged (REF_DIR on the include path)
// so that its static __device__ criteria, range functions and kernels can be
// called directly, and exports plain C entry points for the tests.  The
// checker evaluates one explicit box per thread with the reference's own code;
// the per-box body mirrors the family kernel's innermost loop.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <iostream>
#include <queue>
#include <vector>
#include <csignal>

// output bits per box: bit k = the reference's k-th handle_* returned false;
// 0x20 = empty box after tightening, 0x40 = the fit check fired, 0x80 = trap()
enum : unsigned char { RC_EMPTY = 0x20, RC_FIT = 0x40, RC_TRAP = 0x80 };

#define RC_CHECK(x)                                                               \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            std::fprintf(stderr, "refcheck: %s -> %s\n", #x, cudaGetErrorString(e_)); \
            return 2;                                                             \
        }                                                                         \
    } while (0)

// Runs `kern` over n boxes (SoA host arrays lo/hi of `dims` rows), one box per
// thread, with the trap shim's per-thread slots attached.
template <class Kern>
static int rc_run_boxes(Kern kern, int dims, const double* lo, const double* hi, long n, unsigned char* bits) {
    if (n <= 0) return 0;
    double *dlo = nullptr, *dhi = nullptr;
    unsigned char *dbits = nullptr, *dslots = nullptr;
    size_t bytes = sizeof(double) * (size_t)dims * (size_t)n;
    RC_CHECK(cudaMalloc(&dlo, bytes));
    RC_CHECK(cudaMalloc(&dhi, bytes));
    RC_CHECK(cudaMalloc(&dbits, (size_t)n));
    RC_CHECK(cudaMalloc(&dslots, (size_t)n));
    RC_CHECK(cudaMemcpy(dlo, lo, bytes, cudaMemcpyHostToDevice));
    RC_CHECK(cudaMemcpy(dhi, hi, bytes, cudaMemcpyHostToDevice));
    RC_CHECK(cudaMemset(dslots, 0, (size_t)n));
    RC_CHECK(cudaMemcpyToSymbol(algcuda::refcheck::trap_slots, &dslots, sizeof(dslots)));
    const int block = 128;
    long grid = (n + block - 1) / block;
    kern<<<(unsigned)grid, block>>>(dlo, dhi, n, n, dbits, dslots);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    unsigned char* none = nullptr;
    RC_CHECK(cudaMemcpyToSymbol(algcuda::refcheck::trap_slots, &none, sizeof(none)));
    RC_CHECK(cudaMemcpy(bits, dbits, (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(dlo);
    cudaFree(dhi);
    cudaFree(dbits);
    cudaFree(dslots);
    return 0;
}

template <class Kern>
static int rc_run_lattice(Kern kern, int dims, circlepacking::IV outer, const int* sizes, const long* idx, long n,
                          double* lo, double* hi) {
    if (n <= 0) return 0;
    long* didx = nullptr;
    double *dlo = nullptr, *dhi = nullptr;
    size_t bytes = sizeof(double) * (size_t)dims * (size_t)n;
    RC_CHECK(cudaMalloc(&didx, sizeof(long) * (size_t)n));
    RC_CHECK(cudaMalloc(&dlo, bytes));
    RC_CHECK(cudaMalloc(&dhi, bytes));
    RC_CHECK(cudaMemcpy(didx, idx, sizeof(long) * (size_t)n, cudaMemcpyHostToDevice));
    const int block = 128;
    long grid = (n + block - 1) / block;
    kern<<<(unsigned)grid, block>>>(outer, sizes[0], sizes[1], sizes[2], sizes[3], didx, n, dlo, dhi, n);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    RC_CHECK(cudaMemcpy(lo, dlo, bytes, cudaMemcpyDeviceToHost));
    RC_CHECK(cudaMemcpy(hi, dhi, bytes, cudaMemcpyDeviceToHost));
    cudaFree(didx);
    cudaFree(dlo);
    cudaFree(dhi);
    return 0;
}

// One launch of a reference family kernel over one lambda interval, exactly as
// run_kernel_until_no_criticals (run_kernel.cuh:81-84) issues it.
template <class Kern>
static int rc_kernel_once(Kern kern, dim3 grid, dim3 block, double la_lb, double la_ub, double* first, float* ms) {
    using algcuda::Atomic_ordered_double;
    Atomic_ordered_double h;
    h.set(DBL_MAX);
    Atomic_ordered_double* d = nullptr;
    RC_CHECK(cudaMalloc(&d, sizeof(h)));
    RC_CHECK(cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kern<<<grid, block>>>(circlepacking::IV(la_lb, la_ub), d, false);
    cudaEventRecord(e1);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    cudaEventElapsedTime(ms, e0, e1);
    RC_CHECK(cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost));
    *first = h.get();
    cudaFree(d);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

#define RC_BOX_PROLOGUE                                                   \
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;                \
    if (i >= n) return;                                                   \
    using circlepacking::IV;                                              \
    IV la{lo[i], hi[i]};                                                  \
    IV r1_{lo[stride + i], hi[stride + i]};                               \
    IV r2_{lo[2 * stride + i], hi[2 * stride + i]};

#define RC_LATTICE_PROLOGUE(DIMS)                                         \
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;                \
    if (t >= n) return;                                                   \
    using circlepacking::IV;                                              \
    int nn[4] = {n0, n1, n2, n3};                                         \
    int ix[4] = {0, 0, 0, 0};                                             \
    long rem = idx[t];                                                    \
    for (int d = (DIMS)-1; d >= 0; --d) {                                 \
        ix[d] = (int)(rem % nn[d]);                                       \
        rem /= nn[d];                                                     \
    }
