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

/* The six families (one reference kernel each, in the order the reference proves them, lane_packing.cu:32-37). */
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
 * sizes: subdivision count per axis (host array of dims entries).
 * visited: NULL or n bytes, 0 where the kernel never visits the box (end_3d
 * skips empty r3 ranges, end_configuration.cu:225-227). */
cp_status cp_lattice_boxes(int family, double outer_lb, double outer_ub, const int32_t* sizes, const int64_t* index,
                           size_t n, double* lo, double* hi, size_t stride, uint8_t* visited, void* stream);

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


/* ---------------------------------------------------------------- prover handle
 * A handle owns device scratch (worklists, tables, counters) and a stream, so
 * concurrent handles are independent; one handle must not be used from two
 * threads at once.  cp_create makes `device` current for the calling thread. */
typedef struct cp_prover cp_prover;

cp_status cp_create(int device, cp_prover** out);
void cp_destroy(cp_prover* p);

/* The handle's CUDA stream (cudaStream_t as void*): every kernel the handle
 * launches runs on it, so callers can record events around calls. */
void* cp_get_stream(cp_prover* p);

/* Requests that a running cp_prove_family_reference stop after its current
 * launch (the reference's SIGINT handling, run_kernel.cuh:36-59).  Safe to call
 * from a signal handler or another thread. */
void cp_request_interrupt(cp_prover* p);

/* Called by cp_prove_family_reference before each lattice launch with the
 * lambda interval about to be handled (the reference writes that interval to
 * stderr, run_kernel.cuh:79).  cb = NULL removes the callback. */
typedef void (*cp_step_callback)(void* user, double la_lb, double la_ub);
void cp_set_step_callback(cp_prover* p, cp_step_callback cb, void* user);

/* Called by the host-driven refinement (CP_ENGINE_LEVELS) after each chunk with
 * the boxes evaluated so far and the boxes still waiting on all levels: progress
 * reporting for long refinements.  The callback may call cp_request_interrupt,
 * which stops the refinement after this chunk (CP_ERR_INTERRUPTED, resumable).
 * cb = NULL removes it. */
typedef void (*cp_chunk_callback)(void* user, int64_t evaluated, int64_t waiting);
void cp_set_chunk_callback(cp_prover* p, cp_chunk_callback cb, void* user);

/* Split policies for the box refinement. */
typedef enum cp_split_policy {
    CP_SPLIT_UNIFORM = 0, /* bisect every axis (2^dims children) */
    CP_SPLIT_LAMBDA = 1,  /* bisect lambda only (the reference refines lambda only) */
    CP_SPLIT_WIDEST = 2,  /* bisect the axis with the largest relative width */
    CP_SPLIT_LEARNED = 3, /* bisect the axis the learned model picks (trained or loaded model) */
    CP_SPLIT_HYBRID = 4   /* bisect lambda while its width exceeds lambda_scale * (1 - lambda.hi)^2,
                             else the radius widest relative to the lane width 1 - lambda.hi */
} cp_split_policy;

typedef struct cp_refine_opts {
    int32_t family;
    int32_t precision;      /* cp_precision */
    int32_t policy;         /* cp_split_policy */
    int32_t max_depth;      /* a box not proved at this depth is unresolved (<= 250) */
    int32_t seed_sizes[4];  /* lattice seed: subdivisions per axis */
    double seed_lambda[2];  /* outer lambda interval of the lattice seed */
    int64_t level_capacity; /* boxes per level buffer; 0 = 1<<25 */
    int32_t block;          /* threads per block of the level kernel; 0 = 128 */
    int32_t learned_order;  /* 1 = learned criterion order (needs a trained or loaded model) */
    int32_t engine;         /* cp_engine: host-driven level loop or one CUDA graph launch */
    int32_t boxes_per_thread; /* graph engine: boxes a warp lane takes per claim (1..8); 0 = tuned */
    double lambda_scale;    /* CP_SPLIT_HYBRID: lambda target width scale; 0 = 4e-3 */
    int32_t digest;         /* 1 = compute report->digest (per-box verdict identity checks) */
    int32_t seed_parts;     /* cp_refine: > 1 splits the lattice seed into interleaved pieces ... */
    int32_t seed_part;      /* ... and refines piece seed_part only: lattice boxes seed_part + k * seed_parts
                               (one rank's share of the same proof; the pieces' reports add up to the
                               whole seed's, digests included) */
    int32_t reuse;          /* start family: 1 = a child whose radii equal its parent's (every child of a
                               lambda-only split that clipping leaves alone) takes the parent's
                               lambda-independent criterion terms instead of recomputing them (same
                               values bit for bit; 32 B more per box in the levels above the seed);
                               0 = every box computes every term */
} cp_refine_opts;

/* Refinement engines.  CP_ENGINE_LEVELS: the host picks each chunk, launches
 * the level kernel and reads the counters back (one round trip per chunk).
 * CP_ENGINE_GRAPH: the same schedule runs on the device -- a scheduler kernel
 * and a persistent level kernel (warps claim boxes dynamically) inside a CUDA
 * graph WHILE loop -- so a whole refinement is one graph launch; `block`
 * (64, 128, 256, 512, 1024; 0 = tuned) and boxes_per_thread select the
 * kernel shape.  Both engines produce identical reports. */
typedef enum cp_engine { CP_ENGINE_LEVELS = 0, CP_ENGINE_GRAPH = 1 } cp_engine;

typedef struct cp_refine_report {
    int64_t evaluated;       /* boxes evaluated */
    int64_t verdicts[5];     /* evaluated boxes per cp_verdict */
    int64_t unresolved;      /* boxes not proved at max_depth */
    int64_t clipped;         /* children outside the domain, dropped unevaluated */
    int64_t fp32_decided;    /* boxes proved by the FP32 pass */
    int64_t per_depth[64];   /* boxes evaluated per depth (depth >= 63 in the last) */
    int32_t max_depth_seen;
    int32_t launches;
    double device_ms;        /* summed kernel time (CUDA events on the handle's stream) */
    double wall_ms;          /* host wall time of the call */
    int64_t handles_evaluated; /* guarded criteria evaluated in FP64 (DECIDE order) */
    /* with opts->digest: an order-independent 64-bit sum and xor of a hash of
     * every evaluated box's bounds (bit patterns) and verdict.  Two refinements
     * with equal digests evaluated the same boxes with the same verdicts (up to
     * a 2^-64 collision chance); 0 without opts->digest. */
    uint64_t digest[2];
} cp_refine_report;

/* Refines a family's lattice seed until every box is proved / empty or reaches
 * max_depth.  The seed is the family lattice of opts->seed_sizes over
 * opts->seed_lambda (the boxes cp_lattice_boxes returns); not-proved boxes are
 * bisected per opts->policy and each child is clipped to the dependent ranges
 * of its own lambda interval.  Synchronous.  Returns CP_OK when the search ran
 * to completion (check report->unresolved), or an error status. */
cp_status cp_refine(cp_prover* p, const cp_refine_opts* opts, cp_refine_report* report);

/* As cp_refine from explicit device seed boxes (SoA with stride n, depth bytes
 * may be NULL = 0). */
cp_status cp_refine_boxes(cp_prover* p, const cp_refine_opts* opts, const double* lo, const double* hi,
                          const uint8_t* depth, size_t n, cp_refine_report* report);

/* ---------------------------------------------------------------- full-domain proofs
 * The proof of a family over its whole domain (lambda in [0.5, 0.99] and the
 * dependent radius ranges) by the box refinement: the lambda range is cut into
 * seed slabs, each slab is seeded with a lattice (seed_sizes subdivisions of
 * lambda, r1, r2[, r3] over the slab's own dependent ranges, like the
 * reference's lattices) and refined with `policy` (default lambda only, the
 * reference's own refinement rule, run_kernel.cuh:110-127) down to max_depth.
 * The family is proved when no box is left unresolved.  Stands beside the
 * reference's find_critical_intervals_*_configuration() drivers
 * (lane_packing.cu:27-37) for callers that want the adaptive engine. */
typedef struct cp_proof_opts {
    int32_t family;
    int32_t precision;       /* cp_precision */
    int32_t engine;          /* cp_engine */
    int32_t policy;          /* cp_split_policy (CP_SPLIT_LAMBDA recommended) */
    int32_t max_depth;       /* <= 250 */
    int32_t slabs;           /* seed lambda slabs (>= 1) */
    int32_t geometric;       /* 1: 1 - lambda shrinks by a constant factor from slab to slab
                                (narrower slabs toward 0.99, where the needed lambda width shrinks);
                                0: equal widths */
    int32_t seed_sizes[4];   /* lattice subdivisions per slab: lambda, r1, r2[, r3] */
    int64_t level_capacity;  /* 0 = 1 << 24 */
    int32_t digest;          /* 1 = per-box verdict digest in the report */
    int32_t seed_parts;      /* > 1: refine only the interleaved piece seed_part of every slab's lattice */
    int32_t seed_part;       /* (one rank's share of the proof, see cp_refine_opts) */
    int32_t reuse;           /* see cp_refine_opts.reuse (cp_proof_defaults: 0) */
    int32_t slab_radii[32][3]; /* slab k (k < 32): subdivisions of r1, r2, r3 of its seed lattice where
                                  > 0, else seed_sizes[1..3] */
} cp_proof_opts;

typedef struct cp_proof_report {
    int32_t proved;           /* 1: every slab refined with no unresolved box */
    int32_t slabs_done;
    int64_t evaluated;
    int64_t verdicts[5];
    int64_t unresolved;
    int64_t clipped;
    int64_t per_depth[64];
    int32_t max_depth_seen;
    int32_t first_unresolved_slab; /* -1 when none */
    double device_ms, wall_ms;
    uint64_t digest[2];
} cp_proof_report;

/* The library's settings for a family's full-domain proof: lambda-only
 * refinement from the coarsest seed lattice that proves the family (start and
 * start_end_3d: 18 geometric lambda slabs with a radius lattice per slab),
 * graph engine; CP_ERR_INVALID for a bad family. */
cp_status cp_proof_defaults(int family, cp_proof_opts* opts);

/* The proof of one family (opts->family).  Stops between slabs on
 * cp_request_interrupt (CP_ERR_INTERRUPTED, report->slabs_done).  Returns CP_OK
 * when the refinement ran to completion; report->proved tells the outcome. */
cp_status cp_prove_family(cp_prover* p, const cp_proof_opts* opts, cp_proof_report* report);

/* The proofs of all six families in the reference's order (lane_packing.cu:32-37),
 * each with cp_proof_defaults and the given precision and engine; reports:
 * 6 entries.  Returns the first error status, CP_OK otherwise. */
cp_status cp_prove_all(cp_prover* p, int precision, int engine, cp_proof_report* reports);

/* ---------------------------------------------------------------- reference semantics
 * One launch of a family kernel over one lambda interval with the reference's
 * lattice sizes (run_kernel.cuh:81-84): the smallest lambda.lb of a lattice box
 * whose guarded criteria fail, or +inf when none does (the reference returns
 * DBL_MAX).  Lambda slabs are evaluated in increasing order and the search stops
 * at the first slab holding a failing box.  sizes: NULL = the reference's sizes
 * (start_configuration.cu:41-53, middle_configuration.cu:39-42,
 * end_configuration.cu:39-49).  Returns CP_ERR_NOFIT / CP_ERR_TRAP_SITE where
 * the reference kernel would trap (err_box: 8 doubles lo/hi of the box, or NULL). */
cp_status cp_reference_step(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                            double* first_critical, double* err_box);

typedef struct cp_reference_report {
    int32_t proved;          /* 1 when the lambda queue emptied */
    int32_t interrupted;     /* 1 when stopped by cp_request_interrupt */
    int64_t launches;        /* lattice launches (steps) */
    int64_t boxes_evaluated; /* lattice boxes evaluated */
    double remaining[2];     /* first remaining lambda interval when not proved */
    double device_ms;
    double wall_ms;
} cp_reference_report;

/* The reference's refinement loop run_kernel_until_no_criticals
 * (run_kernel.cuh:61-132) over [la_lb, la_ub]: a min-queue of lambda intervals
 * keyed on lb; each step is cp_reference_step; a failing interval continues on
 * [first, ub] or splits at 0.5*(first+ub).  Stops after max_launches (0 = no
 * limit) or on cp_request_interrupt.  trace: NULL or room for 3*max_launches
 * doubles (lb, ub, first) per step. */
cp_status cp_prove_family_reference(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                                    int64_t max_launches, double* trace, cp_reference_report* report);

/* Every failing box of one lattice launch (the reference's output_criticals
 * rerun, run_kernel.cuh:86-108): up to max_boxes records of 8 doubles (lo/hi of
 * la, r1, r2, r3 after tightening, host memory) plus one byte of failed handle
 * bits each.  *count receives the number of failing boxes found. */
cp_status cp_reference_criticals(cp_prover* p, int family, double la_lb, double la_ub, const int32_t* sizes,
                                 size_t max_boxes, double* boxes, uint8_t* handles, size_t* count);

/* Seeded random boxes on a family's domain, for uneven-depth workloads of the
 * refinement engine (no counterpart in the reference).  Box i takes its numbers
 * from a counter-based generator keyed on (seed, i): lambda's centre is uniform
 * in [0.5, 0.99]; each radius's centre is uniform in its dependent range given
 * the axes before it; every axis has a log-uniform width in [2^-20, 2^-4] and is
 * intersected with its range; the depth byte is uniform in 0..max_label, or
 * 0xFF (dropped, counted as clipped by a refinement) when a range is empty.
 * lo, hi: device SoA with stride n; depth: n device bytes.  Synchronous. */
cp_status cp_random_boxes(cp_prover* p, int family, uint64_t seed, int max_label, size_t n, double* lo, double* hi,
                          uint8_t* depth);

/* As cp_refine_boxes with HOST seed buffers (lo/hi SoA with stride n): copies
 * the seeds into the handle's worklist, refines, synchronises. */
cp_status cp_refine_boxes_host(cp_prover* p, const cp_refine_opts* opts, const double* lo, const double* hi,
                               const uint8_t* depth, size_t n, cp_refine_report* report);

/* Host seeds through two staging slots, so that the copy of the next seed set
 * overlaps the refinement of the current one.  cp_stage_boxes_host starts the
 * host-to-device copy of n boxes of `dims` axes (lo/hi SoA with stride n;
 * depth: n bytes or NULL for depth 0) into staging slot 0 or 1 on the handle's
 * copy stream and returns at once; the host buffers must stay untouched until
 * the refinement that uses the slot has returned, and must be page-locked for
 * the copy to overlap.  cp_refine_staged refines the boxes of a slot as
 * cp_refine_boxes_host would (same report), after the slot's copy finished.
 * A slot may be staged again once the refinement that used it has returned. */
cp_status cp_stage_boxes_host(cp_prover* p, int slot, const double* lo, const double* hi, const uint8_t* depth,
                              size_t n, int dims);
cp_status cp_refine_staged(cp_prover* p, const cp_refine_opts* opts, int slot, cp_refine_report* report);

/* Diagnostics: the library's directed division (Newton reciprocal + exact
 * FMA remainders, used for every interval division in place of the
 * reference's __ddiv_rd/__ddiv_ru, interval.cuh:261-310) next to those
 * intrinsics.  a, b: n device doubles; out: 4n device doubles per element
 * (library RD, library RU, __ddiv_rd, __ddiv_ru).  Asynchronous. */
cp_status cp_div_check(const double* a, const double* b, size_t n, double* out, void* stream);

/* Diagnostics: the FP32 pre-pass's directed division (Newton-corrected
 * reciprocal quotient and exact FMA remainder sign) next to the IEEE intrinsics
 * __fdiv_rd / __fdiv_ru it replaces.  a, b: n device floats; out: 4n device
 * floats per element (library RD, library RU, __fdiv_rd, __fdiv_ru). */
cp_status cp_fdiv_check(const float* a, const float* b, size_t n, float* out, void* stream);

/* Diagnostics: measured peak throughput (operations per second, whole device)
 * of the FP64 primitives the criteria use, each run alone with full occupancy
 * and independent chains: rates[0] DFMA, [1] __dadd_rd, [2] __dmul_rd,
 * [3] __ddiv_rd, [4] asin (CUDA libm), [5] FFMA (FP32), [6] the library's
 * directed division as the kernels call it (one shared copy, cp_div_check),
 * [7] the same inlined and seeded from the FP32 reciprocal, [8] inlined with the
 * FP64 reciprocal seed (rates holds 9 doubles).  Synchronous. */
cp_status cp_measure_primitives(int device, double* rates);

/* ---------------------------------------------------------------- resume and checkpoints
 * The reference keeps its only state, the lambda priority queue, in memory and
 * offers no resume (run_kernel.cuh:71); these entry points let a long
 * refinement on a shared machine stop and continue.  A host-driven refinement
 * (CP_ENGINE_LEVELS) stopped by cp_request_interrupt returns CP_ERR_INTERRUPTED
 * between chunks and leaves its remaining boxes and partial counts in the
 * handle.  Any other refinement or reference-step call discards that state. */

/* Continues the interrupted refinement of this handle; the report covers the
 * whole refinement (counts from before the interruption included). */
cp_status cp_refine_resume(cp_prover* p, cp_refine_report* report);

/* Writes the interrupted refinement (options, counters, the boxes left on every
 * level) to a binary file. */
cp_status cp_checkpoint_save(cp_prover* p, const char* path);

/* Reads a checkpoint into this handle (any handle, e.g. in a new process);
 * cp_refine_resume then continues it.  opts: NULL or receives the options of
 * the checkpointed refinement. */
cp_status cp_checkpoint_load(cp_prover* p, const char* path, cp_refine_opts* opts);

/* ---------------------------------------------------------------- autotuning
 * The level kernel is compiled in CP_LEVEL_VARIANTS register/occupancy variants
 * (minimum resident 128-thread blocks per SM 1, 4, 5, 6).  cp_autotune runs
 * opts' refinement once per variant (after one warm-up run) and keeps the
 * fastest for (opts->family, opts->precision) in the handle.  ms: NULL or
 * CP_LEVEL_VARIANTS doubles receiving each variant's kernel time.  Returns the
 * chosen variant in *best. */
#define CP_LEVEL_VARIANTS 4
cp_status cp_autotune(cp_prover* p, const cp_refine_opts* opts, int* best, double* ms);

/* Graph engine autotuner: times opts' refinement (after one warm-up run) for
 * every block size {64, 128, 256, 512, 1024} x boxes per thread {1, 2, 4, 8}
 * and keeps the fastest for (family, precision).  ms: NULL or 20 doubles
 * (row = block size, column = boxes per thread). */
cp_status cp_autotune_graph(cp_prover* p, const cp_refine_opts* opts, int* block, int* boxes_per_thread, double* ms);

/* Selects a level-kernel variant explicitly (0 .. CP_LEVEL_VARIANTS-1). */
cp_status cp_set_level_variant(cp_prover* p, int family, int precision, int variant);

/* ---------------------------------------------------------------- learned proposal model
 * The reference has no learned component: these entry points serve the
 * CP_SPLIT_LEARNED policy and cp_refine_opts.learned_order, which replace the
 * reference's fixed criterion order (e.g. middle_configuration.cu:196-199) and
 * its lambda-only split (run_kernel.cuh:110-127) by per-box proposals.  The
 * model never issues a verdict.  Network per family: 9 box features -> 64 ->
 * 64 -> 8 logits (4 sub-criterion failure logits, 4 split-axis logits),
 * tanh-GELU, BF16 tensor-core products with FP32 accumulation.
 *
 * cp_model_collect runs cp_refine(opts) (plain policy, no learned options)
 * and labels every sample_stride-th box of each evaluated chunk, up to
 * max_records: FULL-mode failure bits and the split axis whose two children
 * are closest to proved (one-level look-ahead).  The records stay in the
 * handle (one family at a time). */
cp_status cp_model_collect(cp_prover* p, const cp_refine_opts* opts, int64_t max_records, int32_t sample_stride,
                           int64_t* n_records);

/* Copies up to cap records to host memory: feats [cap][16] (BF16 values as
 * float), crit (failure bits), axis (-1 = no split label), boxes [cap][8]
 * (lo, hi per axis), depth.  Any pointer may be NULL.  *n = records held. */
cp_status cp_model_records(cp_prover* p, float* feats, uint8_t* crit, int8_t* axis, double* boxes, uint8_t* depth,
                           size_t cap, size_t* n);

/* Trains the family's network on the collected records on the GPU: seeded
 * initialisation and shuffle, batch (a multiple of 64), Adam with learning
 * rate lr; losses: NULL or epochs floats receiving the mean loss per epoch. */
cp_status cp_model_train(cp_prover* p, int family, int epochs, int batch, float lr, uint64_t seed, float* losses);

/* FP32 master parameters (cp_model_param_count() floats: W1 [16][64], b1 [64],
 * W2 [64][64], b2 [64], W3 [64][8], b3 [8]; W rows = inputs). */
int cp_model_param_count(void);
cp_status cp_model_get_params(cp_prover* p, int family, float* params);
cp_status cp_model_set_params(cp_prover* p, int family, const float* params);

/* One forward + backward pass on the GPU over host rows, without an optimiser
 * step: mean loss and its gradient with respect to the parameters (for
 * gradient checks).  feats [n][16] FP32 (rounded to BF16 on the device). */
cp_status cp_model_loss_grad(int family, const float* params, const float* feats, const uint8_t* crit,
                             const int8_t* axis, size_t n, float* loss, float* grad);

/* As cp_model_loss_grad on a chosen training kernel: kind 0 = warp-level BF16
 * mma.sync (64 rows per block), 1 = tcgen05.mma with FP32 accumulators in
 * tensor memory (128 rows per CTA; bounded completion waits, a time-out
 * returns CP_ERR_DEVICE). */
cp_status cp_model_loss_grad_kind(int kind, int family, const float* params, const float* feats, const uint8_t* crit,
                                  const int8_t* axis, size_t n, float* loss, float* grad);

/* The kernel cp_model_train runs: 1 = tcgen05 (default), 0 = mma.sync. */
cp_status cp_model_set_training(cp_prover* p, int kind);

/* The kernel that runs the network for hints and predictions of the
 * host-driven level loop and cp_model_predict: 1 = tcgen05.mma with FP32
 * accumulators in tensor memory, 128 boxes per CTA (default; the same forward
 * pass the graph engine's level kernel runs inline, so both engines take the
 * same learned decisions), 0 = warp-level BF16 mma.sync.  Bounded completion
 * waits; a time-out returns CP_ERR_DEVICE. */
cp_status cp_model_set_inference(cp_prover* p, int kind);

/* Diagnostics: polls per bounded completion wait of the tcgen05 inference
 * kernel (default 4194304).  0 makes every wait time out at once, so a test can
 * reach the kernel's error path: it drains the MMA in flight, frees its tensor
 * memory and the call returns CP_ERR_DEVICE.  cp_model_set_inference clears a
 * recorded time-out. */
cp_status cp_model_set_wait_limit(cp_prover* p, int32_t polls);

/* Network outputs for host boxes (lo/hi SoA, stride n; depth may be NULL):
 * logits [n][8], the chosen split axis and criterion order per box. */
cp_status cp_model_predict(cp_prover* p, int family, const double* lo, const double* hi, const uint8_t* depth,
                           size_t n, float* logits, uint8_t* axis, uint8_t* order);

/* ---------------------------------------------------------------- no allocation
 * This entry point has no counterpart in the reference.
 *
 * Box refinement for callers that cannot let a library allocate device memory:
 * programs that route every device allocation through their own pool or
 * caching allocator, and latency-critical loops where cudaMalloc's implicit
 * device synchronisation is not acceptable.  It runs the same refinement as
 * cp_refine_boxes (same verdicts, same report) but keeps all its scratch --
 * counters, a single-placement table and the level buffers -- in one fixed
 * 32 MiB array compiled into the library (held on every device that uses it
 * until the process exits), and calls no cudaMalloc or cudaFree.
 *   lo, hi, depth: device seed boxes (SoA, stride n; depth may be NULL = 0);
 *   report: host memory, filled on return; the call synchronises `stream`.
 * Limits: n <= CP_STATIC_MAX_SEEDS and max_depth <= CP_STATIC_MAX_DEPTH; larger
 * requests return CP_ERR_CAPACITY (message in cp_last_error_string()).
 * precision: cp_precision; policy: CP_SPLIT_UNIFORM, _LAMBDA or _WIDEST.
 * The first call on each device sets the array up (resolves its address and
 * fills the table with one kernel launch): make that call before any stream
 * capture.  All calls on a device share the array: calls that overlap on the
 * GPU race and must not be issued. */
#define CP_STATIC_MAX_SEEDS 65536
#define CP_STATIC_MAX_DEPTH 6
cp_status cp_refine_boxes_static(int family, int precision, int policy, int max_depth, const double* lo,
                                 const double* hi, const uint8_t* depth, size_t n, cp_refine_report* report,
                                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CP_PROVER_H_ */
