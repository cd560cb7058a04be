// TEST INFRASTRUCTURE ONLY -- include-path shim for the reference's
// algcuda/exit.cuh, used when the reference's device code is compiled into the
// GPU checker (oracle/_ref/).  The reference's trap() executes the PTX trap
// instruction, which kills the CUDA context; on a shared GPU the checker must
// never do that.  This shim records the event instead: a global counter plus a
// per-thread flag for the checker's one-box-per-thread launches.  Execution then
// continues (an out-of-range asin yields NaN); the checker reports such boxes as
// "trap site reached".
#ifndef ALGCUDA_UTILS_EXIT_CUH_INCLUDED_
#define ALGCUDA_UTILS_EXIT_CUH_INCLUDED_

namespace algcuda {
namespace refcheck {
extern __device__ unsigned int trap_count;
extern __device__ unsigned char* trap_slots;
}  // namespace refcheck

inline __device__ void trap() noexcept {
    atomicAdd(&refcheck::trap_count, 1u);
    unsigned char* slots = refcheck::trap_slots;
    if (slots) slots[blockIdx.x * blockDim.x + threadIdx.x] = 1;
}

inline __device__ void assert_trap(const char*, const char*, int) noexcept { trap(); }

inline __device__ void exit() noexcept { asm("exit;\n"); }
}  // namespace algcuda

#define ALGCUDA_ASSERT(expr) ((void)0)

#endif
