// Pieces of the proposal network shared by the model kernels (cp_model.cu) and
// the persistent level kernel that runs the network inline (cp_graph_kernels.cuh):
// sizes and parameter layouts, the box features, and the tcgen05 building
// blocks (shared-memory descriptors, MMA issue and commit, bounded completion
// waits, tensor-memory loads).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace cpb {
namespace tc {

constexpr int NIN = 9, NK = 16, NH = 64, NO = 8;
// flat FP32 parameters: W1 [16][64] (in x out), b1, W2 [64][64], b2, W3 [64][8], b3
constexpr int P_W1 = 0, P_B1 = P_W1 + NK * NH, P_W2 = P_B1 + NH, P_B2 = P_W2 + NH * NH, P_W3 = P_B2 + NH,
              P_B3 = P_W3 + NH * NO, NPARAM = P_B3 + NO;
// BF16 views in the layouts the fragments read: W1T [64][16], W2T [64][64],
// W3T [8][64] (out x in), W2 [64][64], W3 [64][8] (in x out)
constexpr int V_W1T = 0, V_W2T = V_W1T + NH * NK, V_W3T = V_W2T + NH * NH, V_W2 = V_W3T + NO * NH,
              V_W3 = V_W2 + NH * NH, NVIEW = V_W3 + NH * NO;
constexpr float kGeluC = 0.7978845608028654f;

using bf16 = __nv_bfloat16;

// Inference GELU: the hardware tanh approximation (tanh.approx.f32, one MUFU
// operation; maximum relative error about 2^-11), which is below BF16 resolution.
__device__ __forceinline__ float gelu_fast(float x) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(kGeluC * (x + 0.044715f * x * x * x)));
    return 0.5f * x * (1.0f + t);
}

// The same features in single precision (inference): the relative width is
// clamped at 2^-64, far inside FP32 range, so FP32 log2 loses nothing at BF16
// resolution.
template <int D>
__device__ __forceinline__ void box_features_fast(const double* lo, const double* hi, int depth, float* f) {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        if (d < D) {
            const float a = d == 0 ? 0.5f : 0.0f, inv = d == 0 ? (1.0f / 0.49f) : 4.0f;
            const float c = (float)(0.5 * (lo[d] + hi[d]));
            const float w = fmaxf((float)(hi[d] - lo[d]) * inv, 5.421010862427522e-20f);  // 2^-64
            f[2 * d] = (c - a) * inv * 2.0f - 1.0f;
            f[2 * d + 1] = __log2f(w) * (1.0f / 16.0f) + 1.0f;
        } else {
            f[2 * d] = 0.f;
            f[2 * d + 1] = 0.f;
        }
    }
    f[8] = (float)depth / 32.0f;
#pragma unroll
    for (int k = 9; k < 16; ++k) f[k] = 0.f;
}

constexpr int kTcRows = 128;

// element offset of (row, k) in a K-major core-matrix tile with K columns
__device__ __forceinline__ int cm_off(int row, int k, int K) {
    return (row >> 3) * (K * 8) + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Writes N values (N a multiple of 8) of one row of a K-major core-matrix tile,
// from column k0 (a multiple of 8): each group of 8 columns of a row is 16
// contiguous bytes, written as one 16-byte store of 8 BF16 values (round to
// nearest even, as __float2bfloat16_rn).
template <int N>
__device__ __forceinline__ void put_row_bf16(bf16* tile, int row, int k0, int K, const float* v) {
#pragma unroll
    for (int g = 0; g < N / 8; ++g) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(v[8 * g + 2 * q], v[8 * g + 2 * q + 1]);  // .x: lower column
            w[q] = *reinterpret_cast<const uint32_t*>(&h);
        }
        *reinterpret_cast<uint4*>(tile + cm_off(row, k0 + 8 * g, K)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}
// Hidden-layer epilogue of 32 accumulators of one row: bias + GELU, written as
// BF16 to columns k0..k0+31 of the next operand tile (K = NH).  The biases are
// read into registers before any store, so the 32 independent chains overlap.
__device__ __forceinline__ void gelu_row32(bf16* tile, int row, int k0, const uint32_t* r, const float* bias) {
    float v[32];
#pragma unroll
    for (int c = 0; c < 32; c += 4) {
        const float4 b = *reinterpret_cast<const float4*>(bias + k0 + c);
        v[c] = __uint_as_float(r[c]) + b.x;
        v[c + 1] = __uint_as_float(r[c + 1]) + b.y;
        v[c + 2] = __uint_as_float(r[c + 2]) + b.z;
        v[c + 3] = __uint_as_float(r[c + 3]) + b.w;
    }
#pragma unroll
    for (int c = 0; c < 32; ++c) v[c] = gelu_fast(v[c]);
    put_row_bf16<32>(tile, row, k0, NH, v);
}
// shared-memory matrix descriptor (no swizzle, K-major), Blackwell version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
constexpr int kTcWaitLimit = 1 << 22;  // default polls of a bounded completion wait
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, int limit = kTcWaitLimit) {
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Block-collective completion wait: thread 0 alone polls the mbarrier (so the
// block's other warps take no issue slots from co-resident warps while the
// product runs) and returns 1 when the phase completed within `limit` polls;
// the caller makes the result block-uniform with __syncthreads_and, whose
// barrier orders the other threads after thread 0's observation, and issues
// tcgen05.fence::after_thread_sync before reading the accumulators.
__device__ __forceinline__ int tc_wait_one(uint32_t mbar, uint32_t phase, int limit) {
    return threadIdx.x == 0 ? (mbar_wait(mbar, phase, limit) ? 1 : 0) : 1;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_ld64(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------------ inline forward pass
// The network's forward pass for the 128 threads of a CTA (one box per thread),
// for kernels that run it inline.  Every layer's accumulators land in the same
// 64 tensor-memory columns: each is read back before the next product is
// issued, so a CTA holds only 64 columns.
constexpr uint32_t kNetCols = 64;

struct NetSmem {
    bf16 a[kTcRows * NH];  // operand tile of the current layer (K = 16 or 64)
    bf16 w1[NH * NK];      // W1^T: N = 64, K = 16
    bf16 w2[NH * NH];      // W2^T: N = 64, K = 64
    bf16 w3[16 * NH];      // W3^T padded to N = 16, K = 64
    float b1[NH], b2[NH], b3[16];
    unsigned long long mbar;
    uint32_t tmem;
    uint32_t phase;
};

// Stages the weights, initialises the completion barrier and allocates the
// tensor memory.  All 128 threads call it; a __syncthreads() must follow
// before net_forward.
__device__ __forceinline__ void net_setup(NetSmem& s, const bf16* __restrict__ views, const float* __restrict__ master) {
    const int tid = threadIdx.x;
    for (int i = tid; i < NH * NK; i += kTcRows) s.w1[cm_off(i / NK, i % NK, NK)] = views[V_W1T + i];
    for (int i = tid; i < NH * NH; i += kTcRows) s.w2[cm_off(i / NH, i % NH, NH)] = views[V_W2T + i];
    for (int i = tid; i < 16 * NH; i += kTcRows) {
        const int n = i / NH, k = i % NH;
        s.w3[cm_off(n, k, NH)] = n < NO ? views[V_W3T + n * NH + k] : __float2bfloat16(0.f);
    }
    for (int i = tid; i < NH; i += kTcRows) {
        s.b1[i] = master[P_B1 + i];
        s.b2[i] = master[P_B2 + i];
    }
    if (tid < 16) s.b3[tid] = tid < NO ? master[P_B3 + tid] : 0.f;
    if (tid == 0) {
        s.phase = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((tid >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kNetCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

// One forward pass: f = this thread's 16 features, z = its 8 logits.  Block-
// collective (all 128 threads).  Returns false (block-uniformly) when a
// completion wait ran out; net_teardown then drains the product in flight.
__device__ __forceinline__ bool net_forward(NetSmem& s, const float* f, float* z, int wait_limit) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    put_row_bf16<NK>(s.a, tid, 0, NK, f);
    const uint32_t mbar = smem_u32(&s.mbar);
    uint32_t r[32];
    for (int layer = 0; layer < 3; ++layer) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        const uint32_t tmem = s.tmem;
        const uint32_t phase = s.phase;
        if (tid == 0) {
            const uint32_t a = smem_u32(s.a);
            if (layer == 0) {
                tc_mma(tmem, sdesc(a, 128, NK * 16), sdesc(smem_u32(s.w1), 128, NK * 16), tc_idesc(NH), 0);
            } else {
                const uint32_t w = smem_u32(layer == 1 ? s.w2 : s.w3);
#pragma unroll
                for (int ks = 0; ks < NH / 16; ++ks)
                    tc_mma(tmem, sdesc(a + 256 * ks, 128, NH * 16), sdesc(w + 256 * ks, 128, NH * 16),
                           tc_idesc(layer == 1 ? NH : 16), ks > 0 ? 1u : 0u);
            }
            tc_commit(mbar);
        }
        const bool ok = __syncthreads_and(tc_wait_one(mbar, phase, wait_limit)) != 0;  // block-uniform
        tc_fence_after();
        if (!ok) return false;  // s.phase still names the pending phase
        __syncthreads();        // every thread has read s.phase
        if (tid == 0) s.phase = phase ^ 1u;
        if (layer < 2) {
            // the product has completed, so its operand tile is dead: each thread
            // writes the next layer's row as soon as it has read its accumulators
            const float* bias = layer == 0 ? s.b1 : s.b2;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                tc_ld32(tmem + lane_base + 32u * half, r);
                gelu_row32(s.a, tid, 32 * half, r, bias);
            }
        } else {
            tc_ld16(tmem + lane_base, r);
#pragma unroll
            for (int k = 0; k < NO; ++k) z[k] = __uint_as_float(r[k]) + s.b3[k];
        }
    }
    tc_fence_before();
    __syncthreads();  // the logits are read before the next pass writes the columns
    tc_fence_after();
    return true;
}

// Frees the tensor memory; after a failed pass first waits (bounded) for the
// product still in flight.  All 128 threads call it.
__device__ __forceinline__ void net_teardown(NetSmem& s, bool ok) {
    if (!ok) mbar_wait(smem_u32(&s.mbar), s.phase);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(kNetCols) : "memory");
}

}  // namespace tc
}  // namespace cpb
