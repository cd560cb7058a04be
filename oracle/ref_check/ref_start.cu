// TEST INFRASTRUCTURE ONLY -- checker TU around the reference's
// lane_packing/start_configuration.cu (start, start+end 2-disk and 3-disk).
#include <algcuda/exit.cuh>
#include "start_configuration.cu"
#include "ref_check.cuh"

using namespace circlepacking;
using namespace circlepacking::lane_packing;

// start_configuration.cu:126-162 for one box
static __global__ void rc_eval_start(const double* lo, const double* hi, long n, long stride, unsigned char* bits,
                                     unsigned char* slots) {
    RC_BOX_PROLOGUE
    IV r3{lo[3 * stride + i], hi[3 * stride + i]};
    IV r2 = r2_;
    r2.tighten_lb(r3.get_lb());
    IV r1 = r1_;
    r1.tighten_lb(r2.get_lb());
    if (la.empty() || r1.empty() || r2.empty() || r3.empty()) { bits[i] = RC_EMPTY; return; }
    unsigned char b = 0;
    if (__dmul_ru(2.0, r1.get_ub()) >= __dadd_rd(1.0, -la.get_ub())) b |= RC_FIT;
    IV a12 = collision_angle_outer_inner(la, r1, r2);
    IV a13 = collision_angle_outer_outer(r1, r3);
    IV a23 = collision_angle_inner_outer(la, r2, r3);
    UB case1 = (a12 + a23 > a13);
    if (possibly(case1) && !handle_case_1(la, r1, r2, a12)) b |= 1;
    if (possibly(!case1) && !handle_case_2(la, r1, r2, r3, a13)) b |= 2;
    if (slots[i]) b |= RC_TRAP;
    bits[i] = b;
}

// start_configuration.cu:200-212 for one box
static __global__ void rc_eval_start_end_2d(const double* lo, const double* hi, long n, long stride,
                                            unsigned char* bits, unsigned char* slots) {
    RC_BOX_PROLOGUE
    IV r2 = r2_;
    IV r1 = r1_;
    r1.tighten_lb(r2.get_lb());
    if (la.empty() || r1.empty() || r2.empty()) { bits[i] = RC_EMPTY; return; }
    unsigned char b = 0;
    if (!handle_2d_case(la, r1, r2)) b |= 1;
    if (slots[i]) b |= RC_TRAP;
    bits[i] = b;
}

// start_configuration.cu:277-295 for one box
static __global__ void rc_eval_start_end_3d(const double* lo, const double* hi, long n, long stride,
                                            unsigned char* bits, unsigned char* slots) {
    RC_BOX_PROLOGUE
    IV r3{lo[3 * stride + i], hi[3 * stride + i]};
    IV r2 = r2_;
    r2.tighten_lb(r3.get_lb());
    IV r1 = r1_;
    r1.tighten_lb(r2.get_lb());
    if (la.empty() || r1.empty() || r2.empty() || r3.empty()) { bits[i] = RC_EMPTY; return; }
    unsigned char b = 0;
    if (!handle_3d_case(la, r1, r2, r3)) b |= 1;
    if (slots[i]) b |= RC_TRAP;
    bits[i] = b;
}

// start_configuration.cu:115-125 (loop heads) for explicit lattice coordinates
static __global__ void rc_lattice_start(IV outer, int n0, int n1, int n2, int n3, const long* idx, long n, double* lo,
                                        double* hi, long stride) {
    RC_LATTICE_PROLOGUE(4)
    IV la = get_subinterval(outer, ix[0], n0);
    IV r1 = get_subinterval(compute_r1_range(la), ix[1], n1);
    IV r2 = get_subinterval(compute_r2_range(la, r1), ix[2], n2);
    IV r3 = get_subinterval(compute_r3_range(la, r1, r2), ix[3], n3);
    IV ax[4] = {la, r1, r2, r3};
    for (int d = 0; d < 4; ++d) { lo[d * stride + t] = ax[d].get_lb(); hi[d * stride + t] = ax[d].get_ub(); }
}
static __global__ void rc_lattice_start_end_2d(IV outer, int n0, int n1, int n2, int n3, const long* idx, long n,
                                               double* lo, double* hi, long stride) {
    RC_LATTICE_PROLOGUE(3)
    IV la = get_subinterval(outer, ix[0], n0);
    IV r1 = get_subinterval(compute_r1_range(la), ix[1], n1);
    IV r2 = get_subinterval(compute_r2_range_2d(la, r1), ix[2], n2);
    IV ax[3] = {la, r1, r2};
    for (int d = 0; d < 3; ++d) { lo[d * stride + t] = ax[d].get_lb(); hi[d * stride + t] = ax[d].get_ub(); }
}
static __global__ void rc_lattice_start_end_3d(IV outer, int n0, int n1, int n2, int n3, const long* idx, long n,
                                               double* lo, double* hi, long stride) {
    RC_LATTICE_PROLOGUE(4)
    IV la = get_subinterval(outer, ix[0], n0);
    IV r1 = get_subinterval(compute_r1_range(la), ix[1], n1);
    IV r2 = get_subinterval(compute_r2_range(la, r1), ix[2], n2);
    IV r3 = get_subinterval(compute_r3_range_3d(la, r1, r2), ix[3], n3);
    IV ax[4] = {la, r1, r2, r3};
    for (int d = 0; d < 4; ++d) { lo[d * stride + t] = ax[d].get_lb(); hi[d * stride + t] = ax[d].get_ub(); }
}

extern "C" int refc_eval_boxes_start(int fam, const double* lo, const double* hi, long n, unsigned char* bits) {
    if (fam == 0) return rc_run_boxes(rc_eval_start, 4, lo, hi, n, bits);
    if (fam == 1) return rc_run_boxes(rc_eval_start_end_2d, 3, lo, hi, n, bits);
    if (fam == 2) return rc_run_boxes(rc_eval_start_end_3d, 4, lo, hi, n, bits);
    return 1;
}

extern "C" int refc_lattice_start(int fam, double olb, double oub, const int* sizes, const long* idx, long n,
                                  double* lo, double* hi) {
    IV outer(olb, oub);
    if (fam == 0) return rc_run_lattice(rc_lattice_start, 4, outer, sizes, idx, n, lo, hi);
    if (fam == 1) return rc_run_lattice(rc_lattice_start_end_2d, 3, outer, sizes, idx, n, lo, hi);
    if (fam == 2) return rc_run_lattice(rc_lattice_start_end_3d, 4, outer, sizes, idx, n, lo, hi);
    return 1;
}

// start_configuration.cu:217-225, 300-303: the reference's grid/block per family
extern "C" int refc_kernel_once_start(int fam, double la_lb, double la_ub, double* first, float* ms) {
    if (fam == 0)
        return rc_kernel_once(kernel_find_critical_intervals_start_configuration, dim3(la_parallel, r1_parallel),
                              dim3(r2_parallel, r3_parallel), la_lb, la_ub, first, ms);
    if (fam == 1)
        return rc_kernel_once(kernel_find_critical_intervals_start_end_configuration_2d,
                              dim3(la_parallel_2d, r1_parallel_2d), dim3(r2_parallel_2d), la_lb, la_ub, first, ms);
    if (fam == 2)
        return rc_kernel_once(kernel_find_critical_intervals_start_end_configuration_3d, dim3(la_parallel, r1_parallel),
                              dim3(r2_parallel, r3_parallel), la_lb, la_ub, first, ms);
    return 1;
}
