// TEST INFRASTRUCTURE ONLY -- checker TU around the reference's
// lane_packing/middle_configuration.cu.
#include <algcuda/exit.cuh>
#include "middle_configuration.cu"
#include "ref_check.cuh"

using namespace circlepacking;
using namespace circlepacking::lane_packing;

// middle_configuration.cu:166-201 for one box; the fit check (a trap in the
// reference kernel) is recorded as RC_FIT instead.
static __global__ void rc_eval_middle(const double* lo, const double* hi, long n, long stride, unsigned char* bits,
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
    if (!handle_case_1_1(la, r1, r2, r3)) b |= 1;
    if (!handle_case_2_1(la, r1, r2, r3)) b |= 2;
    if (slots[i]) b |= RC_TRAP;
    bits[i] = b;
}

// middle_configuration.cu:157-168 (loop heads)
static __global__ void rc_lattice_middle(IV outer, int n0, int n1, int n2, int n3, const long* idx, long n, double* lo,
                                         double* hi, long stride) {
    RC_LATTICE_PROLOGUE(4)
    IV la = get_subinterval(outer, ix[0], n0);
    IV r1 = get_subinterval(compute_r1_range(la), ix[1], n1);
    IV r2 = get_subinterval(compute_r2_range(la, r1), ix[2], n2);
    IV r3 = get_subinterval(compute_r3_range(la, r1, r2), ix[3], n3);
    IV ax[4] = {la, r1, r2, r3};
    for (int d = 0; d < 4; ++d) { lo[d * stride + t] = ax[d].get_lb(); hi[d * stride + t] = ax[d].get_ub(); }
}

extern "C" int refc_eval_boxes_middle(int fam, const double* lo, const double* hi, long n, unsigned char* bits) {
    if (fam == 3) return rc_run_boxes(rc_eval_middle, 4, lo, hi, n, bits);
    return 1;
}

extern "C" int refc_lattice_middle(int fam, double olb, double oub, const int* sizes, const long* idx, long n,
                                   double* lo, double* hi) {
    if (fam == 3) return rc_run_lattice(rc_lattice_middle, 4, IV(olb, oub), sizes, idx, n, lo, hi);
    return 1;
}

// middle_configuration.cu:207-212
extern "C" int refc_kernel_once_middle(int fam, double la_lb, double la_ub, double* first, float* ms) {
    if (fam == 3)
        return rc_kernel_once(kernel_find_critical_intervals_middle_configuration, dim3(la_parallel, r1_parallel),
                              dim3(r2_parallel, r3_parallel), la_lb, la_ub, first, ms);
    return 1;
}
