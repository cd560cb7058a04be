/*
 * cp_prover.h -- C ABI of the B200 lane-packing prover.
 *
 * Drop-in boundary for the subinterval search of phillip-keldenich/circlepacking
 * (paths below are relative to the reference's code/ directory).  The reference
 * exposes the path only as argument-less C++ functions and a kernel contract:
 *
 *   void circlepacking::lane_packing::find_critical_intervals();        lane_packing.cu:32-37
 *   void find_critical_intervals_{start,start_end,middle,end}_configuration();
 *                                                                       lane_packing.cu:27-30
 *   bool run_kernel_until_no_criticals(K, IV outer_la, dim3, dim3);     run_kernel.cuh:61-132
 *   __global__ K(IV outer_la, Atomic_ordered_double*, bool);            e.g. middle_configuration.cu:156
 *
 * This header replaces them with plain C entry points: integer status codes, no
 * exceptions, no device trap, no printf from hot kernels.  Device pointers are
 * owned by the caller and work is asynchronous on the given stream unless the
 * function says otherwise; `stream` is a cudaStream_t passed as void* (NULL =
 * the legacy default stream).  A C++ shim (circlepacking_b200/csrc/
 * cp_reference_shim.cpp) defines the reference's argument-less functions on
 * top of this ABI, so the reference's prover.cpp links against it unchanged.
 *
 * Boxes are stored structure-of-arrays: axis d of box i is lo[d*stride + i],
 * hi[d*stride + i]; axes are (lambda, r1, r2) for the 2-disk families and
 * (lambda, r1, r2, r3) for the 3-disk families.  A "raw" box is a lattice box
 * before the per-box tightening r2.lo >= r3.lo, r1.lo >= r2.lo.
 */
#ifndef CP_PROVER_H_
#define CP_PROVER_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference throws std::system_error on CUDA API failures
 * (algcuda/cuda-cpp-wrapper/include/algcuda/error.hpp:84-100) and executes a
 * device trap on invariant violations (algcuda/cuda-utils/cuh/include/algcuda/exit.cuh:28-31). */
typedef enum cp_status {
    CP_OK = 0,
    CP_ERR_INVALID = 1,      /* bad argument */
    CP_ERR_CUDA = 2,         /* CUDA runtime error, see cp_last_error_string() */
    CP_ERR_NOMEM = 3,        /* device allocation failed */
    CP_ERR_CAPACITY = 4,     /* worklist capacity exceeded */
    CP_ERR_DEVICE = 5,       /* a kernel raised its error flag (bounded wait expired, bad index) */
    CP_ERR_TRAP_SITE = 6,    /* a box reached a reference trap site (reference: device trap) */
    CP_ERR_NOFIT = 7,        /* fit check fired where the reference traps (middle/end kernels) */
    CP_ERR_INTERRUPTED = 8,  /* stopped by cp_request_interrupt() (reference: SIGINT, run_kernel.cuh:36-108) */
    CP_ERR_NOT_PROVED = 9,   /* the search ended with unresolved boxes / lambda intervals */
    CP_ERR_NO_DEVICE = 10    /* no CUDA device, or the library's kernels cannot run on it */
} cp_status;

/* The six families (one reference kernel each, SURVEY order). */
typedef enum cp_family {
    CP_START = 0,        /* start_configuration.cu:114-167 */
    CP_START_END_2D = 1, /* start_configuration.cu:190-215 */
    CP_START_END_3D = 2, /* start_configuration.cu:267-298 */
    CP_MIDDLE = 3,       /* middle_configuration.cu:156-205 */
    CP_END_2D = 4,       /* end_configuration.cu:103-146 */
    CP_END_3D = 5        /* end_configuration.cu:212-268 */
} cp_family;

/* Per-box verdicts.  The reference never materialises one: its kernels reduce
 * the minimum lambda.lb over failing boxes (atomic_float.hpp:45-47). */
typedef enum cp_verdict {
    CP_PROVED = 0,   /* every guarded criterion holds */
    CP_CRITICAL = 1, /* some sub-criterion fails (mask bits 0..5) */
    CP_NOFIT = 2,    /* fit check fired in middle/end (reference traps there) */
    CP_EMPTY = 3,    /* an axis is empty after tightening (end_configuration.cu:222-234 skips) */
    CP_ERROR = 4     /* a reference trap site was reached (collision_angles.cu:59-101, interval.cuh:617-621) */
} cp_verdict;

/* Fail-mask bits beside the sub-criterion bits 0..5 */
#define CP_MASK_FIT 0x40u
#define CP_MASK_TRAP 0x80u

typedef enum cp_precision {
    CP_FP64 = 0,           /* FP64 directed rounding, bit-identical to the reference */
    CP_FP32_PREFILTER = 1  /* FP32 enclosure pass issues PROVED; every other box is re-evaluated in FP64 */
} cp_precision;

typedef enum cp_eval_mode {
    CP_EVAL_FULL = 0,  /* every sub-criterion evaluated: complete mask */
    CP_EVAL_DECIDE = 1 /* stop at the first failing handle; PROVED/EMPTY identical to FULL */
} cp_eval_mode;

/* Number of axes of a family's boxes (3 or 4), or -1. */
int cp_family_dims(int family);

/* Number of sub-criteria (mask bits) of a family, or -1. */
int cp_family_criteria(int family);

/* Static description of a status code. */
const char* cp_status_string(int status);

/* Text of the last CUDA error seen by this thread ("" if none). */
const char* cp_last_error_string(void);

/* Library version string. */
const char* cp_version(void);

/* Per-box evaluation of n raw boxes on the device.  Replaces the innermost
 * loop body of the family kernels (e.g. middle_configuration.cu:166-201), one
 * verdict per box instead of the reference's min-reduction.
 *   precision: cp_precision; mode: cp_eval_mode
 *   verdict, mask: n bytes each (device); order: NULL or n bytes (DECIDE mode:
 *   bit 0 = evaluate the second handle first); trace: NULL or n*16 doubles,
 *   (lhs, rhs) of each sub-criterion, FULL mode only, untouched where a
 *   guard skipped the sub-criterion.  Asynchronous on `stream`. */
cp_status cp_eval_boxes(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                        size_t stride, uint8_t* verdict, uint8_t* mask, const uint8_t* order, double* trace,
                        void* stream);

/* As cp_eval_boxes, with HOST buffers: copies in, evaluates, copies out and
 * synchronises (the reference's blocking cudaMemcpy pattern, memory.cpp:27-47). */
cp_status cp_eval_boxes_host(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                             uint8_t* verdict, uint8_t* mask);

/* Boxes of a family lattice: for each linear index idx (axis order
 * lambda, r1, r2[, r3], last fastest) the raw box the reference's kernel loop
 * builds with get_subinterval (subintervals.hpp:31-42) over its dependent
 * ranges (compute_r*_range, e.g. middle_configuration.cu:66-84).
 * sizes: subdivision count per axis (host array of dims entries). */
cp_status cp_lattice_boxes(int family, double outer_lb, double outer_ub, const int32_t* sizes, const int64_t* index,
                           size_t n, double* lo, double* hi, size_t stride, void* stream);

/* lower_bound_radius_single_placement(lb_lambda) for n values
 * (lower_bound_radius_single_placement.cu:26-61).  Device arrays. */
cp_status cp_single_placement(const double* lb_lambda, size_t n, double* out, void* stream);

/* Diagnostics: one geometric primitive on n explicit interval arguments.
 * kind 0 collision_angle_inner_inner(la,ra,rb), 1 outer_inner(la,ra,rb),
 * 2 inner_outer(la,ra,rb), 3 outer_outer(ra,rb), 4 semicircle_angle_outer(r),
 * 5 semicircle_angle_inner(la,r)  (collision_angles.cu:119-246).
 * args: 6*n doubles, rows lb0,ub0,lb1,ub1,lb2,ub2; out: lb[n] then ub[n];
 * trap: n bytes (1 = a trap site was reached).  Device arrays. */
cp_status cp_eval_primitive(int kind, const double* args, size_t n, double* out, uint8_t* trap, void* stream);

/* Diagnostics: outward-padded asin bounds (interval.cuh:420-438).  Device arrays. */
cp_status cp_asin_pad(const double* x, size_t n, double* rd, double* ru, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CP_PROVER_H_ */
