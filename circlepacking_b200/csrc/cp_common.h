// Internal helpers shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include "cp_prover.h"

namespace cpb {
struct LatticeSpec;
}

// Threads per block of the per-box evaluation kernels.
constexpr int kEvalBlock = 128;

// Records a CUDA error for cp_last_error_string() and returns `status`.
cp_status cp_record_cuda_error(cudaError_t e, cp_status status);

// Records a formatted message for cp_last_error_string() and returns `status`.
cp_status cp_fail(cp_status status, const char* fmt, ...);

// Checks for a launch error right after a kernel launch.
cp_status cp_check_launch();

// Launches the per-box evaluation (see cp_eval_boxes).
cp_status cp_launch_eval(int family, int precision, int mode, const double* lo, const double* hi, size_t n,
                         size_t stride, uint8_t* verdict, uint8_t* mask, const uint8_t* order, double* trace,
                         cudaStream_t st);

// Single placement bound of the lower end of every lambda slab of a lattice.
cp_status cp_launch_slab_single(const cpb::LatticeSpec& s, double* out, cudaStream_t st);
