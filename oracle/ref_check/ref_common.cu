// TEST INFRASTRUCTURE ONLY -- checker TU: the trap shim's state, the
// reference's geometric primitives (collision_angles.cu,
// lower_bound_radius_single_placement.cu) and asin padding (interval.cuh:420-438)
// on explicit inputs, and the per-family dispatch of the other TUs.
#include <algcuda/exit.cuh>
#include "operations.cuh"
#include <algcuda/atomic_float.hpp>
#include "ref_check.cuh"

namespace algcuda {
namespace refcheck {
__device__ unsigned int trap_count = 0;
__device__ unsigned char* trap_slots = nullptr;
}  // namespace refcheck
}  // namespace algcuda

using namespace circlepacking;
using namespace circlepacking::lane_packing;

// kind: 0 inner_inner(la,ra,rb), 1 outer_inner(la,ra,rb), 2 inner_outer(la,ra,rb),
// 3 outer_outer(ra,rb), 4 semicircle_outer(r), 5 semicircle_inner(la,r)
static __global__ void rc_primitive(int kind, const double* in, long n, double* out, unsigned char* slots) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    IV a0{in[0 * n + i], in[1 * n + i]}, a1{in[2 * n + i], in[3 * n + i]}, a2{in[4 * n + i], in[5 * n + i]};
    IV r{0.0, 0.0};
    switch (kind) {
    case 0: r = collision_angle_inner_inner(a0, a1, a2); break;
    case 1: r = collision_angle_outer_inner(a0, a1, a2); break;
    case 2: r = collision_angle_inner_outer(a0, a1, a2); break;
    case 3: r = collision_angle_outer_outer(a0, a1); break;
    case 4: r = semicircle_angle_outer(a0); break;
    case 5: r = semicircle_angle_inner(a0, a1); break;
    }
    out[i] = r.get_lb();
    out[n + i] = r.get_ub();
}

static __global__ void rc_single(const double* lam, long n, double* out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = lower_bound_radius_single_placement(lam[i]);
}

static __global__ void rc_asin(const double* x, long n, double* rd, double* ru) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        rd[i] = algcuda::detail::dasin_rd(x[i]);
        ru[i] = algcuda::detail::dasin_ru(x[i]);
    }
}

extern "C" {
int refc_eval_boxes_start(int, const double*, const double*, long, unsigned char*);
int refc_eval_boxes_middle(int, const double*, const double*, long, unsigned char*);
int refc_eval_boxes_end(int, const double*, const double*, long, unsigned char*);
int refc_lattice_start(int, double, double, const int*, const long*, long, double*, double*);
int refc_lattice_middle(int, double, double, const int*, const long*, long, double*, double*);
int refc_lattice_end(int, double, double, const int*, const long*, long, double*, double*);
int refc_kernel_once_start(int, double, double, double*, float*);
int refc_kernel_once_middle(int, double, double, double*, float*);
int refc_kernel_once_end(int, double, double, double*, float*);

// Per-box handle results of the reference's own criteria for n explicit boxes
// (host arrays lo/hi, dims x n).  bits as in ref_check.cuh.
int refc_eval_boxes(int fam, const double* lo, const double* hi, long n, unsigned char* bits) {
    if (fam <= 2) return refc_eval_boxes_start(fam, lo, hi, n, bits);
    if (fam == 3) return refc_eval_boxes_middle(fam, lo, hi, n, bits);
    return refc_eval_boxes_end(fam, lo, hi, n, bits);
}

// Boxes of a family lattice, generated by the reference's own get_subinterval
// and compute_r*_range on the device.
int refc_lattice_boxes(int fam, double olb, double oub, const int* sizes, const long* idx, long n, double* lo,
                       double* hi) {
    if (fam <= 2) return refc_lattice_start(fam, olb, oub, sizes, idx, n, lo, hi);
    if (fam == 3) return refc_lattice_middle(fam, olb, oub, sizes, idx, n, lo, hi);
    return refc_lattice_end(fam, olb, oub, sizes, idx, n, lo, hi);
}

// One launch of the reference's own family kernel over [la_lb, la_ub]; returns
// the first problematic lambda (DBL_MAX when none) and the kernel time.
int refc_kernel_once(int fam, double la_lb, double la_ub, double* first, float* ms) {
    if (fam <= 2) return refc_kernel_once_start(fam, la_lb, la_ub, first, ms);
    if (fam == 3) return refc_kernel_once_middle(fam, la_lb, la_ub, first, ms);
    return refc_kernel_once_end(fam, la_lb, la_ub, first, ms);
}

int refc_primitive(int kind, const double* in, long n, double* out, unsigned char* trap) {
    if (n <= 0) return 0;
    double *din = nullptr, *dout = nullptr;
    unsigned char* dslots = nullptr;
    RC_CHECK(cudaMalloc(&din, sizeof(double) * 6 * (size_t)n));
    RC_CHECK(cudaMalloc(&dout, sizeof(double) * 2 * (size_t)n));
    RC_CHECK(cudaMalloc(&dslots, (size_t)n));
    RC_CHECK(cudaMemcpy(din, in, sizeof(double) * 6 * (size_t)n, cudaMemcpyHostToDevice));
    RC_CHECK(cudaMemset(dslots, 0, (size_t)n));
    RC_CHECK(cudaMemcpyToSymbol(algcuda::refcheck::trap_slots, &dslots, sizeof(dslots)));
    rc_primitive<<<(unsigned)((n + 127) / 128), 128>>>(kind, din, n, dout, dslots);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    unsigned char* none = nullptr;
    RC_CHECK(cudaMemcpyToSymbol(algcuda::refcheck::trap_slots, &none, sizeof(none)));
    RC_CHECK(cudaMemcpy(out, dout, sizeof(double) * 2 * (size_t)n, cudaMemcpyDeviceToHost));
    if (trap) RC_CHECK(cudaMemcpy(trap, dslots, (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(din);
    cudaFree(dout);
    cudaFree(dslots);
    return 0;
}

int refc_single_placement(const double* lam, long n, double* out) {
    if (n <= 0) return 0;
    double *din = nullptr, *dout = nullptr;
    RC_CHECK(cudaMalloc(&din, sizeof(double) * (size_t)n));
    RC_CHECK(cudaMalloc(&dout, sizeof(double) * (size_t)n));
    RC_CHECK(cudaMemcpy(din, lam, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
    rc_single<<<(unsigned)((n + 127) / 128), 128>>>(din, n, dout);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    RC_CHECK(cudaMemcpy(out, dout, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(din);
    cudaFree(dout);
    return 0;
}

int refc_asin_pad(const double* x, long n, double* rd, double* ru) {
    if (n <= 0) return 0;
    double *dx = nullptr, *drd = nullptr, *dru = nullptr;
    RC_CHECK(cudaMalloc(&dx, sizeof(double) * (size_t)n));
    RC_CHECK(cudaMalloc(&drd, sizeof(double) * (size_t)n));
    RC_CHECK(cudaMalloc(&dru, sizeof(double) * (size_t)n));
    RC_CHECK(cudaMemcpy(dx, x, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
    rc_asin<<<(unsigned)((n + 127) / 128), 128>>>(dx, n, drd, dru);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaDeviceSynchronize());
    RC_CHECK(cudaMemcpy(rd, drd, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    RC_CHECK(cudaMemcpy(ru, dru, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(dx);
    cudaFree(drd);
    cudaFree(dru);
    return 0;
}

unsigned refc_trap_count_reset(void) {
    unsigned h = 0, z = 0;
    if (cudaMemcpyFromSymbol(&h, algcuda::refcheck::trap_count, sizeof(h)) != cudaSuccess) return 0xFFFFFFFFu;
    cudaMemcpyToSymbol(algcuda::refcheck::trap_count, &z, sizeof(z));
    return h;
}
}  // extern "C"
