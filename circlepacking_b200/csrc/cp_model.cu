// Learned proposal model: per box, which guarded criterion to evaluate first and
// which axis to bisect.  The reference has no learned component; the model only
// reorders work and chooses splits -- every verdict is still issued by the
// interval kernels (cp_families.cuh), so soundness does not depend on it.
//
// Network (one per family): 9 features -> 64 -> 64 -> 8 logits, tanh-GELU.
//   logits 0..3  failure of sub-criterion k (binary cross-entropy, k < K)
//   logits 4..7  split axis (softmax cross-entropy over the family's axes)
// Weights and activations enter the tensor cores as BF16 (mma.sync m16n8k16,
// FP32 accumulation); master weights, Adam moments and biases stay FP32.
//
// Features of a box (computed in FP64, rounded to BF16): per axis d < dims the
// centre mapped to [-1, 1] over the axis' nominal range and
// log2(max(width / range, 2^-64)) / 16 + 1; then depth / 32.  Ranges: lambda [0.5, 0.99],
// radii [0, 0.25].
//
// Training records come from the prover's own refinement (cp_model_collect):
// sampled boxes of every evaluated chunk, labelled with their FULL-mode failure
// bits and with the axis whose two children are closest to proved (one-level
// look-ahead; a child's badness is 1 + the relative deficit of its worst
// failing criterion, 0 when it is proved, empty or outside the domain).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "cp_common.h"
#include "cp_engine.h"
#include "cp_level.cuh"
#include "cp_tc.cuh"

using namespace cpb;

namespace {

using namespace cpb::tc;

// shared-memory pitches (elements) chosen so fragment loads are bank-conflict free
constexpr int PK = 24, PH = 72;
constexpr int kRowsPerWarp = 16, kTrainWarps = 4, kTrainRows = kRowsPerWarp * kTrainWarps;


__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    uint32_t u;
    memcpy(&u, &v, 4);
    return u;
}
__device__ __forceinline__ uint32_t ld32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D += A (16x16, row-major) * B (16x8, column-major); BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float gelu(float x) {
    const float t = tanhf(kGeluC * (x + 0.044715f * x * x * x));
    return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanhf(kGeluC * (x + 0.044715f * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * 0.044715f * x * x);
}

// Model features of one box (see the file comment); f[9..15] = 0.
template <int D>
__device__ __forceinline__ void box_features(const double* lo, const double* hi, int depth, float* f) {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        if (d < D) {
            const double a = d == 0 ? 0.5 : 0.0, rng = d == 0 ? 0.49 : 0.25;
            const double c = 0.5 * (lo[d] + hi[d]);
            const double w = fmax((hi[d] - lo[d]) / rng, 5.421010862427522e-20);  // 2^-64
            f[2 * d] = (float)((c - a) / rng * 2.0 - 1.0);
            f[2 * d + 1] = (float)(log2(w) / 16.0 + 1.0);
        } else {
            f[2 * d] = 0.f;
            f[2 * d + 1] = 0.f;
        }
    }
    f[8] = (float)depth / 32.0f;
#pragma unroll
    for (int k = 9; k < 16; ++k) f[k] = 0.f;
}


// Shared-memory copies of the forward weights.
struct FwdSmem {
    bf16 w1t[NH * PK];
    bf16 w2t[NH * PH];
    bf16 w3t[NO * PH];
    float b1[NH], b2[NH], b3[NO];
};

__device__ void load_fwd(FwdSmem& s, const bf16* __restrict__ views, const float* __restrict__ master) {
    for (int i = threadIdx.x; i < NH * NK; i += blockDim.x) s.w1t[(i / NK) * PK + i % NK] = views[V_W1T + i];
    for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) s.w2t[(i / NH) * PH + i % NH] = views[V_W2T + i];
    for (int i = threadIdx.x; i < NO * NH; i += blockDim.x) s.w3t[(i / NH) * PH + i % NH] = views[V_W3T + i];
    for (int i = threadIdx.x; i < NH; i += blockDim.x) {
        s.b1[i] = master[P_B1 + i];
        s.b2[i] = master[P_B2 + i];
    }
    for (int i = threadIdx.x; i < NO; i += blockDim.x) s.b3[i] = master[P_B3 + i];
}

// Forward pass of one warp's 16 rows.  x: the rows' features, BF16 [16][PK] in
// shared memory.  Keeps the pre-activations (for the backward pass) and the
// logits in accumulator layout: z[0..1] row g, cols 2t..2t+1; z[2..3] row g+8.
struct Acts {
    float h1[8][4], h2[8][4], z[4];
    uint32_t g1[4][4], g2[4][4];
};

template <bool FAST>
__device__ __forceinline__ float act(float x) {
    return FAST ? gelu_fast(x) : gelu(x);
}

template <bool FAST>
__device__ __forceinline__ void forward16(const FwdSmem& s, const bf16* x, Acts& A) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint32_t ax[4] = {ld32(x + g * PK + 2 * t), ld32(x + (g + 8) * PK + 2 * t), ld32(x + g * PK + 2 * t + 8),
                            ld32(x + (g + 8) * PK + 2 * t + 8)};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        float acc[4] = {s.b1[c], s.b1[c + 1], s.b1[c], s.b1[c + 1]};
        mma16816(acc, ax, ld32(s.w1t + (8 * j + g) * PK + 2 * t), ld32(s.w1t + (8 * j + g) * PK + 2 * t + 8));
#pragma unroll
        for (int e = 0; e < 4; ++e) A.h1[j][e] = acc[e];
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        A.g1[kt][0] = pack2(act<FAST>(A.h1[2 * kt][0]), act<FAST>(A.h1[2 * kt][1]));
        A.g1[kt][1] = pack2(act<FAST>(A.h1[2 * kt][2]), act<FAST>(A.h1[2 * kt][3]));
        A.g1[kt][2] = pack2(act<FAST>(A.h1[2 * kt + 1][0]), act<FAST>(A.h1[2 * kt + 1][1]));
        A.g1[kt][3] = pack2(act<FAST>(A.h1[2 * kt + 1][2]), act<FAST>(A.h1[2 * kt + 1][3]));
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        float acc[4] = {s.b2[c], s.b2[c + 1], s.b2[c], s.b2[c + 1]};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt)
            mma16816(acc, A.g1[kt], ld32(s.w2t + (8 * j + g) * PH + 16 * kt + 2 * t),
                     ld32(s.w2t + (8 * j + g) * PH + 16 * kt + 2 * t + 8));
#pragma unroll
        for (int e = 0; e < 4; ++e) A.h2[j][e] = acc[e];
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        A.g2[kt][0] = pack2(act<FAST>(A.h2[2 * kt][0]), act<FAST>(A.h2[2 * kt][1]));
        A.g2[kt][1] = pack2(act<FAST>(A.h2[2 * kt][2]), act<FAST>(A.h2[2 * kt][3]));
        A.g2[kt][2] = pack2(act<FAST>(A.h2[2 * kt + 1][0]), act<FAST>(A.h2[2 * kt + 1][1]));
        A.g2[kt][3] = pack2(act<FAST>(A.h2[2 * kt + 1][2]), act<FAST>(A.h2[2 * kt + 1][3]));
    }
    float acc[4] = {s.b3[2 * t], s.b3[2 * t + 1], s.b3[2 * t], s.b3[2 * t + 1]};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
        mma16816(acc, A.g2[kt], ld32(s.w3t + g * PH + 16 * kt + 2 * t), ld32(s.w3t + g * PH + 16 * kt + 2 * t + 8));
#pragma unroll
    for (int e = 0; e < 4; ++e) A.z[e] = acc[e];
}

// Writes the two BF16 halves of a packed register into a transposed staging
// tile: T[col][row] and T[col + 1][row].
__device__ __forceinline__ void put_t(bf16* T, int pitch, int col, int row, uint32_t packed) {
    __nv_bfloat162 v;
    memcpy(&v, &packed, 4);
    T[col * pitch + row] = v.x;
    T[(col + 1) * pitch + row] = v.y;
}

// ------------------------------------------------------------------ training
struct TrainSmem {
    FwdSmem f;
    bf16 w2[NH * PH];  // W2 (in x out) for dG1 = dH2 W2^T
    bf16 w3[NH * NO];  // W3 (in x out) for dG2 = dZ W3^T
    bf16 xt[NK * PH];  // staged transposes over the block's 64 rows
    bf16 g1t[NH * PH];
    bf16 g2t[NH * PH];
    bf16 dzt[NO * PH];
    bf16 dh2t[NH * PH];
    bf16 dh1t[NH * PH];
    bf16 x[kTrainWarps][kRowsPerWarp * PK];
    float loss[kTrainWarps];
};

struct TrainArgs {
    const bf16* feats;   // [n][16]
    const uint8_t* crit; // failure bits per row
    const int8_t* axis;  // best axis per row, -1 = none
    size_t row0, rows;   // this batch: rows [row0, row0 + rows)
    size_t n;            // total records (rows beyond n are padding)
    int K, D;
    float inv_batch;
    const bf16* views;
    const float* master;
    float* grad;
    float* loss;         // accumulated mean loss (may be null)
    int* step;           // incremented once per launch (Adam's step count)
};

// One fused forward + backward pass over 64 rows per block; weight and bias
// gradients are reduced across blocks with FP32 atomics into a.grad.
__global__ void __launch_bounds__(kTrainWarps * 32) k_train_step(TrainArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& s = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.step) atomicAdd(a.step, 1);
    load_fwd(s.f, a.views, a.master);
    for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) s.w2[(i / NH) * PH + i % NH] = a.views[V_W2 + i];
    for (int i = threadIdx.x; i < NH * NO; i += blockDim.x) s.w3[i] = a.views[V_W3 + i];
    const size_t brow = a.row0 + (size_t)blockIdx.x * kTrainRows;  // block's first row
    // features of the block's rows (zero beyond the batch / the record set)
    for (int i = threadIdx.x; i < kTrainRows * NK; i += blockDim.x) {
        const int r = i / NK, k = i % NK;
        const size_t row = brow + r;
        const bool ok = row < a.row0 + a.rows && row < a.n;
        const bf16 v = ok ? a.feats[row * NK + k] : __float2bfloat16(0.f);
        s.x[r / kRowsPerWarp][(r % kRowsPerWarp) * PK + k] = v;
        s.xt[k * PH + r] = v;
    }
    __syncthreads();

    Acts A;
    forward16<false>(s.f, s.x[warp], A);
    const int rw = kRowsPerWarp * warp;  // warp's first row within the block
    // stage G1, G2 transposed for the weight gradients
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        put_t(s.g1t, PH, 16 * kt + 2 * t, rw + g, A.g1[kt][0]);
        put_t(s.g1t, PH, 16 * kt + 2 * t, rw + g + 8, A.g1[kt][1]);
        put_t(s.g1t, PH, 16 * kt + 8 + 2 * t, rw + g, A.g1[kt][2]);
        put_t(s.g1t, PH, 16 * kt + 8 + 2 * t, rw + g + 8, A.g1[kt][3]);
        put_t(s.g2t, PH, 16 * kt + 2 * t, rw + g, A.g2[kt][0]);
        put_t(s.g2t, PH, 16 * kt + 2 * t, rw + g + 8, A.g2[kt][1]);
        put_t(s.g2t, PH, 16 * kt + 8 + 2 * t, rw + g, A.g2[kt][2]);
        put_t(s.g2t, PH, 16 * kt + 8 + 2 * t, rw + g + 8, A.g2[kt][3]);
    }

    // ---- loss and dZ (accumulator layout)
    float dz[4] = {0.f, 0.f, 0.f, 0.f};
    float lsum = 0.f;
    float o[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) o[e] = __shfl_xor_sync(0xffffffffu, A.z[e], 1);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const size_t row = brow + rw + g + 8 * half;
        const bool valid = row < a.row0 + a.rows && row < a.n;
        const float z0 = A.z[2 * half], z1 = A.z[2 * half + 1];
        if (!valid) continue;
        if (t < 2) {
            const unsigned bits = a.crit[row];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int k = 2 * t + e;
                if (k < a.K) {
                    const float z = e ? z1 : z0;
                    const float y = (float)((bits >> k) & 1u);
                    const float sp = fmaxf(z, 0.f) + log1pf(expf(-fabsf(z)));
                    lsum += sp - y * z;
                    dz[2 * half + e] = (1.f / (1.f + expf(-z)) - y) * a.inv_batch;
                }
            }
        } else {
            const int lab = a.axis[row];
            if (lab >= 0) {
                // this lane holds axes 2(t-2), 2(t-2)+1; the partner lane the other two
                const int ax0 = 2 * (t - 2), px0 = 2 * (3 - t);
                float v[4];
                v[ax0] = z0;
                v[ax0 + 1] = z1;
                v[px0] = o[2 * half];
                v[px0 + 1] = o[2 * half + 1];
                float m = -INFINITY;
#pragma unroll
                for (int d = 0; d < 4; ++d)
                    if (d < a.D) m = fmaxf(m, v[d]);
                float ssum = 0.f;
#pragma unroll
                for (int d = 0; d < 4; ++d)
                    if (d < a.D) ssum += expf(v[d] - m);
                if (t == 2) lsum += m + logf(ssum) - v[lab];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int d = ax0 + e;
                    if (d < a.D) dz[2 * half + e] = (expf(v[d] - m) / ssum - (d == lab ? 1.f : 0.f)) * a.inv_batch;
                }
            }
        }
    }
    const uint32_t dzp0 = pack2(dz[0], dz[1]), dzp1 = pack2(dz[2], dz[3]);
    put_t(s.dzt, PH, 2 * t, rw + g, dzp0);
    put_t(s.dzt, PH, 2 * t, rw + g + 8, dzp1);
    // db3
    {
        float c0 = dz[0] + dz[2], c1 = dz[1] + dz[3];
        for (int off = 4; off < 32; off <<= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, off);
            c1 += __shfl_xor_sync(0xffffffffu, c1, off);
        }
        if (g == 0) {
            atomicAdd(&a.grad[P_B3 + 2 * t], c0);
            atomicAdd(&a.grad[P_B3 + 2 * t + 1], c1);
        }
    }

    // ---- dG2 = dZ W3^T (K = 8, zero-padded to 16), dH2 = dG2 * gelu'(H2)
    const uint32_t adz[4] = {dzp0, dzp1, 0u, 0u};
    uint32_t dh2f[4][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(acc, adz, ld32(s.w3 + (8 * j + g) * NO + 2 * t), 0u);
        float dh[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) dh[e] = acc[e] * gelu_grad(A.h2[j][e]);
        const uint32_t p0 = pack2(dh[0], dh[1]), p1 = pack2(dh[2], dh[3]);
        put_t(s.dh2t, PH, 8 * j + 2 * t, rw + g, p0);
        put_t(s.dh2t, PH, 8 * j + 2 * t, rw + g + 8, p1);
        dh2f[j >> 1][(j & 1) * 2 + 0] = p0;
        dh2f[j >> 1][(j & 1) * 2 + 1] = p1;
        float c0 = dh[0] + dh[2], c1 = dh[1] + dh[3];
        for (int off = 4; off < 32; off <<= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, off);
            c1 += __shfl_xor_sync(0xffffffffu, c1, off);
        }
        if (g == 0) {
            atomicAdd(&a.grad[P_B2 + 8 * j + 2 * t], c0);
            atomicAdd(&a.grad[P_B2 + 8 * j + 2 * t + 1], c1);
        }
    }
    // ---- dG1 = dH2 W2^T, dH1 = dG1 * gelu'(H1)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt)
            mma16816(acc, dh2f[kt], ld32(s.w2 + (8 * j + g) * PH + 16 * kt + 2 * t),
                     ld32(s.w2 + (8 * j + g) * PH + 16 * kt + 2 * t + 8));
        float dh[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) dh[e] = acc[e] * gelu_grad(A.h1[j][e]);
        put_t(s.dh1t, PH, 8 * j + 2 * t, rw + g, pack2(dh[0], dh[1]));
        put_t(s.dh1t, PH, 8 * j + 2 * t, rw + g + 8, pack2(dh[2], dh[3]));
        float c0 = dh[0] + dh[2], c1 = dh[1] + dh[3];
        for (int off = 4; off < 32; off <<= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, off);
            c1 += __shfl_xor_sync(0xffffffffu, c1, off);
        }
        if (g == 0) {
            atomicAdd(&a.grad[P_B1 + 8 * j + 2 * t], c0);
            atomicAdd(&a.grad[P_B1 + 8 * j + 2 * t + 1], c1);
        }
    }
    // loss: warp sum, then one atomic per block
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if (lane == 0) s.loss[warp] = lsum;
    __syncthreads();
    if (threadIdx.x == 0 && a.loss) {
        float l = 0.f;
        for (int w = 0; w < kTrainWarps; ++w) l += s.loss[w];
        if (l != 0.f) atomicAdd(a.loss, l * a.inv_batch);
    }

    // ---- weight gradients over the block's 64 rows (K = rows)
    // dW3 [64][8] = G2^T dZ: warp w owns input rows 16w..16w+15
    {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const int m0 = 16 * warp;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            const int k = 16 * kt + 2 * t;
            const uint32_t af[4] = {ld32(s.g2t + (m0 + g) * PH + k), ld32(s.g2t + (m0 + g + 8) * PH + k),
                                    ld32(s.g2t + (m0 + g) * PH + k + 8), ld32(s.g2t + (m0 + g + 8) * PH + k + 8)};
            mma16816(acc, af, ld32(s.dzt + g * PH + k), ld32(s.dzt + g * PH + k + 8));
        }
        atomicAdd(&a.grad[P_W3 + (m0 + g) * NO + 2 * t], acc[0]);
        atomicAdd(&a.grad[P_W3 + (m0 + g) * NO + 2 * t + 1], acc[1]);
        atomicAdd(&a.grad[P_W3 + (m0 + g + 8) * NO + 2 * t], acc[2]);
        atomicAdd(&a.grad[P_W3 + (m0 + g + 8) * NO + 2 * t + 1], acc[3]);
    }
    // dW2 [64][64] = G1^T dH2: warp w owns input rows 16w..16w+15
    {
        const int m0 = 16 * warp;
        uint32_t af[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            const int k = 16 * kt + 2 * t;
            af[kt][0] = ld32(s.g1t + (m0 + g) * PH + k);
            af[kt][1] = ld32(s.g1t + (m0 + g + 8) * PH + k);
            af[kt][2] = ld32(s.g1t + (m0 + g) * PH + k + 8);
            af[kt][3] = ld32(s.g1t + (m0 + g + 8) * PH + k + 8);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                const int k = 16 * kt + 2 * t;
                mma16816(acc, af[kt], ld32(s.dh2t + (8 * j + g) * PH + k), ld32(s.dh2t + (8 * j + g) * PH + k + 8));
            }
            const int c = 8 * j + 2 * t;
            atomicAdd(&a.grad[P_W2 + (m0 + g) * NH + c], acc[0]);
            atomicAdd(&a.grad[P_W2 + (m0 + g) * NH + c + 1], acc[1]);
            atomicAdd(&a.grad[P_W2 + (m0 + g + 8) * NH + c], acc[2]);
            atomicAdd(&a.grad[P_W2 + (m0 + g + 8) * NH + c + 1], acc[3]);
        }
    }
    // dW1 [16][64] = X^T dH1: warp w owns output columns 16w..16w+15
    {
        uint32_t af[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            const int k = 16 * kt + 2 * t;
            af[kt][0] = ld32(s.xt + g * PH + k);
            af[kt][1] = ld32(s.xt + (g + 8) * PH + k);
            af[kt][2] = ld32(s.xt + g * PH + k + 8);
            af[kt][3] = ld32(s.xt + (g + 8) * PH + k + 8);
        }
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const int j = 2 * warp + jj;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                const int k = 16 * kt + 2 * t;
                mma16816(acc, af[kt], ld32(s.dh1t + (8 * j + g) * PH + k), ld32(s.dh1t + (8 * j + g) * PH + k + 8));
            }
            const int c = 8 * j + 2 * t;
            if (g < NIN) {
                atomicAdd(&a.grad[P_W1 + g * NH + c], acc[0]);
                atomicAdd(&a.grad[P_W1 + g * NH + c + 1], acc[1]);
            }
            if (g + 8 < NIN) {
                atomicAdd(&a.grad[P_W1 + (g + 8) * NH + c], acc[2]);
                atomicAdd(&a.grad[P_W1 + (g + 8) * NH + c + 1], acc[3]);
            }
        }
    }
}

// Writes the BF16 views of the FP32 master weights.
__device__ __forceinline__ void write_views(int i, float w, bf16* views) {
    const bf16 b = __float2bfloat16_rn(w);
    if (i < P_B1) {
        const int k = i / NH, n = i % NH;
        views[V_W1T + n * NK + k] = b;
    } else if (i >= P_W2 && i < P_B2) {
        const int r = i - P_W2, k = r / NH, n = r % NH;
        views[V_W2T + n * NH + k] = b;
        views[V_W2 + k * NH + n] = b;
    } else if (i >= P_W3 && i < P_B3) {
        const int r = i - P_W3, k = r / NO, n = r % NO;
        views[V_W3T + n * NH + k] = b;
        views[V_W3 + k * NO + n] = b;
    }
}

__global__ void k_views(const float* __restrict__ master, bf16* __restrict__ views) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x)
        write_views(i, master[i], views);
}

// Adam (bias-corrected); clears the gradient and refreshes the BF16 views.
__global__ void k_adam(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                       float* __restrict__ grad, bf16* __restrict__ views, const int* __restrict__ step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int tstep = *step;
    const float c1 = 1.f - powf(b1, (float)tstep), c2 = 1.f - powf(b2, (float)tstep);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        grad[i] = 0.f;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float w = master[i];
        if (!(i >= P_W1 + NIN * NH && i < P_B1))  // padded input rows stay zero
            w -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        master[i] = w;
        write_views(i, w, views);
    }
}

// ------------------------------------------------------------------ inference
struct InferArgs {
    BoxList in;
    size_t begin, count;
    const bf16* views;
    const float* master;
    uint8_t* axis;     // per box, indexed from `begin` (may be null)
    uint8_t* order;    // per box (may be null)
    float* logits;     // [count][8] (may be null)
};

struct InferSmem {
    FwdSmem f;
    bf16 x[4][kRowsPerWarp * PK];
    float z[4][kRowsPerWarp * NO];
};

// The criterion order and split axis of boxes [begin, begin+count): each warp
// runs the network on 16 boxes at a time.
template <int FAM>
__global__ void __launch_bounds__(128) k_infer(InferArgs a) {
    constexpr int D = family_dims(FAM);
    __shared__ InferSmem s;
    load_fwd(s.f, a.views, a.master);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const size_t groups = (a.count + kRowsPerWarp - 1) / kRowsPerWarp;
    for (size_t grp = (size_t)blockIdx.x * 4 + warp; grp < groups; grp += (size_t)gridDim.x * 4) {
        const size_t j0 = grp * kRowsPerWarp;
        if (lane < kRowsPerWarp) {
            float f[16];
            const size_t j = j0 + lane;
            if (j < a.count) {
                const size_t i = a.begin + j;
                double lo[4], hi[4];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    lo[d] = a.in.lo[d * a.in.cap + i];
                    hi[d] = a.in.hi[d * a.in.cap + i];
                }
                const int depth = a.in.depth[i];
                box_features_fast<D>(lo, hi, depth == 0xFF ? 0 : depth, f);
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) f[k] = 0.f;
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) s.x[warp][lane * PK + k] = __float2bfloat16_rn(f[k]);
        }
        __syncwarp();
        Acts A;
        forward16<true>(s.f, s.x[warp], A);
        s.z[warp][g * NO + 2 * t] = A.z[0];
        s.z[warp][g * NO + 2 * t + 1] = A.z[1];
        s.z[warp][(g + 8) * NO + 2 * t] = A.z[2];
        s.z[warp][(g + 8) * NO + 2 * t + 1] = A.z[3];
        __syncwarp();
        if (lane < kRowsPerWarp && j0 + lane < a.count) {
            const float* z = s.z[warp] + lane * NO;
            const size_t j = j0 + lane;
            int ord = 0;
            if (FAM == F_MIDDLE)
                ord = fmaxf(z[2], z[3]) > fmaxf(z[0], z[1]) ? 1 : 0;
            else if (FAM == F_END_2D || FAM == F_END_3D)
                ord = z[1] > z[0] ? 1 : 0;
            int ax = 0;
            float best = z[4];
#pragma unroll
            for (int d = 1; d < D; ++d)
                if (z[4 + d] > best) {
                    best = z[4 + d];
                    ax = d;
                }
            if (a.order) a.order[j] = (uint8_t)ord;
            if (a.axis) a.axis[j] = (uint8_t)ax;
            if (a.logits)
                for (int k = 0; k < NO; ++k) a.logits[j * NO + k] = z[k];
        }
        __syncwarp();
    }
}


// ------------------------------------------------------------------ inference on tcgen05
// The same forward pass on the 5th-generation tensor cores: a CTA takes 128
// boxes (one per thread), stages their features and the weights in shared
// memory in the canonical K-major core-matrix layout (8 rows x 16 bytes per
// core matrix; LBO = 128 B between core matrices along K, SBO = K * 16 B
// between 8-row groups), and one thread issues tcgen05.mma (M = 128, N = 64 or
// 16, K = 16 per instruction, BF16 in, FP32 accumulators in tensor memory).
// Every thread reads its box's row back with tcgen05.ld, applies bias and
// GELU, and writes the next layer's operand tile.  Waits on the MMA-completion
// mbarrier are bounded: on time-out the kernel raises *err, waits (bounded)
// once more, frees its tensor memory and returns.
constexpr uint32_t kTcCols = 128;  // tensor-memory columns per CTA: [0, 64) hidden, [64, 80) logits

struct TcSmem {
    bf16 a[kTcRows * NH];  // activation tile (K <= 64)
    bf16 w1[NH * NK];      // W1^T: N = 64 rows, K = 16
    bf16 w2[NH * NH];      // W2^T: 64 x 64
    bf16 w3[16 * NH];      // W3^T padded to N = 16 rows, K = 64
    float b1[NH], b2[NH], b3[16];
    unsigned long long mbar;
    uint32_t tmem;
};

struct TcArgs {
    InferArgs a;
    int* err;        // raised when an MMA-completion wait times out
    int wait_limit;  // polls per completion wait (0: every wait times out at once)
};

template <int FAM>
__global__ void __launch_bounds__(kTcRows) k_infer_tc(TcArgs ta) {
    constexpr int D = family_dims(FAM);
    __shared__ __align__(1024) TcSmem s;
    const InferArgs& a = ta.a;
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights and biases, staged once per CTA
    for (int i = tid; i < NH * NK; i += kTcRows) s.w1[cm_off(i / NK, i % NK, NK)] = a.views[V_W1T + i];
    for (int i = tid; i < NH * NH; i += kTcRows) s.w2[cm_off(i / NH, i % NH, NH)] = a.views[V_W2T + i];
    for (int i = tid; i < 16 * NH; i += kTcRows) {
        const int n = i / NH, k = i % NH;
        s.w3[cm_off(n, k, NH)] = n < NO ? a.views[V_W3T + n * NH + k] : __float2bfloat16(0.f);
    }
    for (int i = tid; i < NH; i += kTcRows) {
        s.b1[i] = a.master[P_B1 + i];
        s.b2[i] = a.master[P_B2 + i];
    }
    if (tid < 16) s.b3[tid] = tid < NO ? a.master[P_B3 + tid] : 0.f;
    const uint32_t mbar = smem_u32(&s.mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;  // this warp's quadrant of tensor-memory lanes
    const uint32_t a_addr = smem_u32(s.a), w1_addr = smem_u32(s.w1), w2_addr = smem_u32(s.w2),
                   w3_addr = smem_u32(s.w3);
    uint32_t phase = 0;
    bool ok = true;
    const size_t tiles = (a.count + kTcRows - 1) / kTcRows;
    for (size_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const size_t j = tile * kTcRows + tid;
        // ---- features of this thread's box -> layer-1 operand tile (K = 16)
        {
            float f[16];
            if (j < a.count) {
                const size_t i = a.begin + j;
                double lo[4], hi[4];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    lo[d] = a.in.lo[d * a.in.cap + i];
                    hi[d] = a.in.hi[d * a.in.cap + i];
                }
                const int depth = a.in.depth[i];
                box_features_fast<D>(lo, hi, depth == 0xFF ? 0 : depth, f);
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) f[k] = 0.f;
            }
            put_row_bf16<NK>(s.a, tid, 0, NK, f);
        }
        uint32_t r[64];
#pragma unroll
        for (int layer = 0; layer < 3; ++layer) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                if (layer == 0) {
                    tc_mma(tmem, sdesc(a_addr, 128, NK * 16), sdesc(w1_addr, 128, NK * 16), tc_idesc(NH), 0);
                } else {
                    const uint32_t w_addr = layer == 1 ? w2_addr : w3_addr;
                    const uint32_t d_col = layer == 1 ? 0u : 64u;
                    const uint32_t idesc = tc_idesc(layer == 1 ? NH : 16);
#pragma unroll
                    for (int ks = 0; ks < NH / 16; ++ks)
                        tc_mma(tmem + d_col, sdesc(a_addr + 256 * ks, 128, NH * 16), sdesc(w_addr + 256 * ks, 128, NH * 16),
                               idesc, ks > 0 ? 1u : 0u);
                }
                tc_commit(mbar);
            }
            ok = __syncthreads_and(tc_wait_one(mbar, phase, ta.wait_limit)) != 0;  // block-uniform
            // the parity advances only past a completed phase: after a time-out
            // `phase` still names the pending one, which the drain below waits for
            if (ok) phase ^= 1u;
            tc_fence_after();
            if (!ok) break;
            if (layer < 2) {
                tc_ld64(tmem + lane_base, r);
                const float* bias = layer == 0 ? s.b1 : s.b2;
                tc_fence_before();
                __syncthreads();  // every thread has read its row; the tile may be overwritten
                gelu_row32(s.a, tid, 0, r, bias);
                gelu_row32(s.a, tid, 32, r + 32, bias);
            } else {
                tc_ld16(tmem + lane_base + 64u, r);
            }
        }
        if (!ok) break;
        if (j < a.count) {
            float z[NO];
#pragma unroll
            for (int k = 0; k < NO; ++k) z[k] = __uint_as_float(r[k]) + s.b3[k];
            int ord = 0;
            if (FAM == F_MIDDLE)
                ord = fmaxf(z[2], z[3]) > fmaxf(z[0], z[1]) ? 1 : 0;
            else if (FAM == F_END_2D || FAM == F_END_3D)
                ord = z[1] > z[0] ? 1 : 0;
            int ax = 0;
            float best = z[4];
#pragma unroll
            for (int d = 1; d < D; ++d)
                if (z[4 + d] > best) {
                    best = z[4 + d];
                    ax = d;
                }
            if (a.order) a.order[j] = (uint8_t)ord;
            if (a.axis) a.axis[j] = (uint8_t)ax;
            if (a.logits)
                for (int k = 0; k < NO; ++k) a.logits[j * NO + k] = z[k];
        }
    }
    if (!ok) {
        if (tid == 0) atomicExch(ta.err, 1);
        // bounded: let the MMA still in flight (committed to the pending phase)
        // finish before its tensor memory is freed
        mbar_wait(mbar, phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

// ------------------------------------------------------------------ training on tcgen05
// One fused forward + backward pass of 128 rows per CTA on the 5th-generation
// tensor cores.  Every product runs as tcgen05.mma (M = 128, BF16 operands in
// shared memory in the canonical K-major core-matrix layout, FP32 accumulators
// in tensor memory); each thread owns one row, reads its accumulator row back
// with tcgen05.ld and writes the next operand tiles:
//   H1 = X W1,  H2 = G1 W2,  Z = G2 W3                        (forward)
//   dG2 = dZ W3^T,  dG1 = dH2 W2^T                             (data gradients)
//   dW2 = G1^T dH2,  dW3 = G2^T dZ,  dW1^T = dH1^T X          (weight gradients, K = the 128 rows)
// The weight-gradient products have 64 real output rows; their A tiles are
// 128 rows high with rows 64..127 zero, so every product uses the M = 128
// accumulator layout (row r in tensor-memory lane r).  Gradients of the CTA's
// rows are added to a.grad with FP32 atomics.  Completion waits are bounded: on
// a time-out the kernel raises *err, drains the MMAs in flight, frees its
// tensor memory and returns.
constexpr uint32_t kTtCols = 512;
// accumulator columns (each product's block starts on a multiple of 64 columns)
constexpr uint32_t TT_H1 = 0, TT_H2 = 64, TT_Z = 128, TT_DG2 = 192, TT_DG1 = 256, TT_DW2 = 320, TT_DW3 = 384,
                   TT_DW1 = 448;

struct TtSmem {
    bf16 x[kTcRows * NK];      // A of H1 (K = 16 inputs)
    bf16 xt[NK * kTcRows];     // B of dW1^T (N = 16 inputs, K = 128 rows)
    bf16 g1[kTcRows * NH];     // A of H2
    bf16 g1t[kTcRows * kTcRows];  // A of dW2 (64 hidden units + 64 zero rows, K = 128 rows)
    bf16 g2[kTcRows * NH];     // A of Z
    bf16 g2t[kTcRows * kTcRows];  // A of dW3
    bf16 dz[kTcRows * 16];     // A of dG2 (K = 16: 8 logits, 8 zero)
    bf16 dzt[16 * kTcRows];    // B of dW3 (N = 16, K = 128 rows)
    bf16 dh2[kTcRows * NH];    // A of dG1
    bf16 dh2t[NH * kTcRows];   // B of dW2 (N = 64, K = 128 rows)
    bf16 dh1t[kTcRows * kTcRows];  // A of dW1^T
    bf16 w1t[NH * NK];         // B of H1: W1^T (N = 64, K = 16)
    bf16 w2t[NH * NH];         // B of H2: W2^T
    bf16 w3t[16 * NH];         // B of Z: W3^T padded to N = 16
    bf16 w3[NH * 16];          // B of dG2: W3 (N = 64, K = 16: 8 logits, 8 zero)
    bf16 w2[NH * NH];          // B of dG1: W2 (N = 64, K = 64)
    float b1[NH], b2[NH], b3[16];
    float colsum[NH + NH + 16];  // bias gradients of the CTA's rows: db1, db2, db3
    float loss;
    unsigned long long mbar;
    uint32_t tmem;
};


// D (tensor memory, column dcol) = A (128 x K tile) * B (N x K tile)^T, K = 16 * ksteps
__device__ __forceinline__ void tt_gemm(uint32_t tmem, uint32_t dcol, const bf16* A, const bf16* B, int K, int N) {
    const uint32_t a = smem_u32(A), b = smem_u32(B), sbo = (uint32_t)K * 16u;
    for (int ks = 0; ks < K / 16; ++ks)
        tc_mma(tmem + dcol, sdesc(a + 256u * ks, 128, sbo), sdesc(b + 256u * ks, 128, sbo), tc_idesc(N), ks > 0 ? 1u : 0u);
}

struct TtArgs {
    TrainArgs t;
    int* err;
    int wait_limit;
};

__global__ void __launch_bounds__(kTcRows) k_train_tc(TtArgs ta) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TtSmem& s = *reinterpret_cast<TtSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const TrainArgs& a = ta.t;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (blockIdx.x == 0 && tid == 0 && a.step) atomicAdd(a.step, 1);
    // weights (BF16 views), biases, zero pads
    for (int i = tid; i < NH * NK; i += kTcRows) s.w1t[cm_off(i / NK, i % NK, NK)] = a.views[V_W1T + i];
    for (int i = tid; i < NH * NH; i += kTcRows) {
        s.w2t[cm_off(i / NH, i % NH, NH)] = a.views[V_W2T + i];
        s.w2[cm_off(i / NH, i % NH, NH)] = a.views[V_W2 + i];
    }
    for (int i = tid; i < 16 * NH; i += kTcRows) {
        const int n = i / NH, k = i % NH;
        s.w3t[cm_off(n, k, NH)] = n < NO ? a.views[V_W3T + n * NH + k] : __float2bfloat16(0.f);
        const int i2 = i / 16, o = i % 16;  // W3 as [64 hidden][16 logits, zero padded]
        s.w3[cm_off(i2, o, 16)] = o < NO ? a.views[V_W3 + i2 * NO + o] : __float2bfloat16(0.f);
    }
    for (int i = tid; i < NH; i += kTcRows) {
        s.b1[i] = a.master[P_B1 + i];
        s.b2[i] = a.master[P_B2 + i];
    }
    if (tid < 16) s.b3[tid] = tid < NO ? a.master[P_B3 + tid] : 0.f;
    for (int i = tid; i < NH + NH + 16; i += kTcRows) s.colsum[i] = 0.f;
    if (tid == 0) s.loss = 0.f;
    // rows 64..127 of the weight-gradient A tiles stay zero
    for (int i = tid; i < (kTcRows - NH) * kTcRows; i += kTcRows) {
        const int r = NH + i / kTcRows, k = i % kTcRows;
        s.g1t[cm_off(r, k, kTcRows)] = __float2bfloat16(0.f);
        s.g2t[cm_off(r, k, kTcRows)] = __float2bfloat16(0.f);
        s.dh1t[cm_off(r, k, kTcRows)] = __float2bfloat16(0.f);
    }
    // this thread's row: features
    const size_t row = a.row0 + (size_t)blockIdx.x * kTcRows + tid;
    const bool valid = row < a.row0 + a.rows && row < a.n;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const bf16 v = valid ? a.feats[row * NK + k] : __float2bfloat16(0.f);
        s.x[cm_off(tid, k, NK)] = v;
        s.xt[cm_off(k, tid, kTcRows)] = v;
    }
    const uint32_t mbar = smem_u32(&s.mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTtCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    uint32_t phase = 0;
    bool ok = true;
    uint32_t tmem = 0;
    // one stage: make the operand tiles visible to the tensor cores, issue, wait
    auto stage = [&](int which) -> bool {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        tmem = s.tmem;
        if (tid == 0) {
            switch (which) {
            case 0: tt_gemm(tmem, TT_H1, s.x, s.w1t, NK, NH); break;
            case 1: tt_gemm(tmem, TT_H2, s.g1, s.w2t, NH, NH); break;
            case 2: tt_gemm(tmem, TT_Z, s.g2, s.w3t, NH, 16); break;
            case 3: tt_gemm(tmem, TT_DG2, s.dz, s.w3, 16, NH); break;
            case 4:
                tt_gemm(tmem, TT_DG1, s.dh2, s.w2, NH, NH);
                tt_gemm(tmem, TT_DW2, s.g1t, s.dh2t, kTcRows, NH);
                tt_gemm(tmem, TT_DW3, s.g2t, s.dzt, kTcRows, 16);
                break;
            default: tt_gemm(tmem, TT_DW1, s.dh1t, s.xt, kTcRows, 16); break;
            }
            tc_commit(mbar);
        }
        const bool done = __syncthreads_and(tc_wait_one(mbar, phase, ta.wait_limit)) != 0;  // block-uniform
        if (done) phase ^= 1u;  // after a time-out `phase` names the pending phase (drained below)
        tc_fence_after();
        return done;
    };
    uint32_t r[32], q[32];
    do {
        // ---- forward
        if (!(ok = stage(0))) break;
        for (int c0 = 0; c0 < NH; c0 += 32) {
            tc_ld32(tmem + lane_base + TT_H1 + c0, r);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const bf16 g = __float2bfloat16_rn(gelu(__uint_as_float(r[c]) + s.b1[c0 + c]));
                s.g1[cm_off(tid, c0 + c, NH)] = g;
                s.g1t[cm_off(c0 + c, tid, kTcRows)] = g;
            }
        }
        if (!(ok = stage(1))) break;
        for (int c0 = 0; c0 < NH; c0 += 32) {
            tc_ld32(tmem + lane_base + TT_H2 + c0, r);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const bf16 g = __float2bfloat16_rn(gelu(__uint_as_float(r[c]) + s.b2[c0 + c]));
                s.g2[cm_off(tid, c0 + c, NH)] = g;
                s.g2t[cm_off(c0 + c, tid, kTcRows)] = g;
            }
        }
        if (!(ok = stage(2))) break;
        // ---- loss and dZ of this thread's row
        {
            uint32_t zr[16];
            tc_ld16(tmem + lane_base + TT_Z, zr);
            float z[NO], dz[NO];
#pragma unroll
            for (int k = 0; k < NO; ++k) {
                z[k] = __uint_as_float(zr[k]) + s.b3[k];
                dz[k] = 0.f;
            }
            float l = 0.f;
            if (valid) {
                const unsigned bits = a.crit[row];
                for (int k = 0; k < a.K; ++k) {
                    const float y = (float)((bits >> k) & 1u);
                    l += fmaxf(z[k], 0.f) + log1pf(expf(-fabsf(z[k]))) - y * z[k];
                    dz[k] = (1.f / (1.f + expf(-z[k])) - y) * a.inv_batch;
                }
                const int lab = a.axis[row];
                if (lab >= 0) {
                    float m = -INFINITY;
                    for (int d = 0; d < a.D; ++d) m = fmaxf(m, z[4 + d]);
                    float ssum = 0.f;
                    for (int d = 0; d < a.D; ++d) ssum += expf(z[4 + d] - m);
                    l += m + logf(ssum) - z[4 + lab];
                    for (int d = 0; d < a.D; ++d)
                        dz[4 + d] = (expf(z[4 + d] - m) / ssum - (d == lab ? 1.f : 0.f)) * a.inv_batch;
                }
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const float v = k < NO ? dz[k] : 0.f;
                const bf16 b = __float2bfloat16_rn(v);
                s.dz[cm_off(tid, k, 16)] = b;
                s.dzt[cm_off(k, tid, kTcRows)] = b;
                if (k < NO && v != 0.f) atomicAdd(&s.colsum[NH + NH + k], v);
            }
            for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
            if (lane == 0 && l != 0.f) atomicAdd(&s.loss, l);
        }
        // ---- dH2 = (dZ W3^T) * gelu'(H2)
        if (!(ok = stage(3))) break;
        for (int c0 = 0; c0 < NH; c0 += 32) {
            tc_ld32(tmem + lane_base + TT_DG2 + c0, r);
            tc_ld32(tmem + lane_base + TT_H2 + c0, q);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const float d = __uint_as_float(r[c]) * gelu_grad(__uint_as_float(q[c]) + s.b2[c0 + c]);
                const bf16 b = __float2bfloat16_rn(d);
                s.dh2[cm_off(tid, c0 + c, NH)] = b;
                s.dh2t[cm_off(c0 + c, tid, kTcRows)] = b;
                if (d != 0.f) atomicAdd(&s.colsum[NH + c0 + c], d);
            }
        }
        // ---- dH1 = (dH2 W2^T) * gelu'(H1); dW2 and dW3 in the same stage
        if (!(ok = stage(4))) break;
        for (int c0 = 0; c0 < NH; c0 += 32) {
            tc_ld32(tmem + lane_base + TT_DG1 + c0, r);
            tc_ld32(tmem + lane_base + TT_H1 + c0, q);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const float d = __uint_as_float(r[c]) * gelu_grad(__uint_as_float(q[c]) + s.b1[c0 + c]);
                s.dh1t[cm_off(c0 + c, tid, kTcRows)] = __float2bfloat16_rn(d);
                if (d != 0.f) atomicAdd(&s.colsum[c0 + c], d);
            }
        }
        // dW2 (rows = hidden units 0..63 in lanes 0..63: warps 0 and 1)
        if (warp < 2) {
            for (int c0 = 0; c0 < NH; c0 += 32) {
                tc_ld32(tmem + lane_base + TT_DW2 + c0, r);
#pragma unroll
                for (int c = 0; c < 32; ++c) atomicAdd(&a.grad[P_W2 + tid * NH + c0 + c], __uint_as_float(r[c]));
            }
            uint32_t w3r[16];
            tc_ld16(tmem + lane_base + TT_DW3, w3r);
#pragma unroll
            for (int o = 0; o < NO; ++o) atomicAdd(&a.grad[P_W3 + tid * NO + o], __uint_as_float(w3r[o]));
        }
        if (!(ok = stage(5))) break;
        if (warp < 2) {
            uint32_t w1r[16];
            tc_ld16(tmem + lane_base + TT_DW1, w1r);  // dW1^T row = hidden unit tid, columns = inputs
#pragma unroll
            for (int k = 0; k < NK; ++k) atomicAdd(&a.grad[P_W1 + k * NH + tid], __uint_as_float(w1r[k]));
        }
    } while (0);
    if (!ok) {
        if (tid == 0) atomicExch(ta.err, 1);
        mbar_wait(mbar, phase);  // bounded: the MMAs committed to the pending phase finish first
    } else {
        __syncthreads();
        for (int i = tid; i < NH + NH + 16; i += kTcRows) {
            const float v = s.colsum[i];
            if (v == 0.f) continue;
            if (i < NH)
                atomicAdd(&a.grad[P_B1 + i], v);
            else if (i < 2 * NH)
                atomicAdd(&a.grad[P_B2 + i - NH], v);
            else if (i - 2 * NH < NO)
                atomicAdd(&a.grad[P_B3 + i - 2 * NH], v);
        }
        if (tid == 0 && a.loss && s.loss != 0.f) atomicAdd(a.loss, s.loss * a.inv_batch);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(kTtCols) : "memory");
}

// ------------------------------------------------------------------ trace records
struct LabelArgs {
    BoxList in;
    size_t begin, count;
    size_t stride, phase;  // label boxes j = phase, phase + stride, ... of the chunk
    SingleTable tab;
    bf16* feats;
    uint8_t* crit;
    int8_t* axis;
    double* box;           // [cap][8]: lo/hi interleaved per axis
    uint8_t* depth;
    unsigned long long* count_out;
    size_t cap;
};

// Badness of a box for the look-ahead label: 0 when proved, empty or outside
// the domain; otherwise 1 + the relative deficit of its worst failing criterion.
template <int FAM>
__device__ double badness(const double* lo, const double* hi) {
    double tr[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) tr[k] = 0.0;
    const Verdict v = eval_box<FAM, FULL>(lo, hi, 0, tr);
    if (v.verdict == V_PROVED || v.verdict == V_EMPTY) return 0.0;
    if (v.verdict != V_CRITICAL) return 2.0;
    double worst = 0.0;
    for (int k = 0; k < 6; ++k)
        if (v.mask & (1u << k)) {
            const double lhs = tr[2 * k], rhs = tr[2 * k + 1];
            const double def = (rhs - lhs) / fmax(fabs(rhs), 1e-300);
            if (def > worst) worst = def;
        }
    return 1.0 + fmin(worst, 1.0);
}

template <int FAM>
__global__ void __launch_bounds__(128) k_label(LabelArgs a) {
    constexpr int D = family_dims(FAM);
    const size_t nsel = a.phase < a.count ? (a.count - a.phase + a.stride - 1) / a.stride : 0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nsel; q += (size_t)gridDim.x * blockDim.x) {
        const size_t i = a.begin + a.phase + q * a.stride;
        const int depth = a.in.depth[i];
        if (depth == 0xFF) continue;
        double lo[4], hi[4];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            lo[d] = a.in.lo[d * a.in.cap + i];
            hi[d] = a.in.hi[d * a.in.cap + i];
        }
        const Verdict v = eval_box<FAM, FULL>(lo, hi, 0, nullptr);
        if (v.verdict == V_EMPTY) continue;
        int label = -1;
        if (v.verdict == V_CRITICAL) {
            double best = 1e300, best_w = -1.0;
            for (int ax = 0; ax < D; ++ax) {
                double s = 0.0;
                for (int c = 0; c < 2; ++c) {
                    double clo[4], chi[4];
                    make_child<D>(lo, hi, SPLIT_GIVEN, ax, c, clo, chi);
                    if (clip_child<FAM>(clo, chi, a.tab)) s += badness<FAM>(clo, chi);
                }
                const double w = ax == 0 ? (hi[0] - lo[0]) / fmax(1.0 - hi[0], 1e-300)
                                         : (hi[ax] - lo[ax]) / fmax(hi[ax], 1e-300);
                if (s < best - 1e-12 || (fabs(s - best) <= 1e-12 && w > best_w)) {
                    best = s;
                    best_w = w;
                    label = ax;
                }
            }
        }
        const unsigned long long k = atomicAdd(a.count_out, 1ull);
        if (k >= a.cap) continue;
        float f[16];
        box_features<D>(lo, hi, depth, f);
        for (int j = 0; j < 16; ++j) a.feats[k * NK + j] = __float2bfloat16_rn(f[j]);
        a.crit[k] = (uint8_t)(v.mask & 0x0F);
        a.axis[k] = (int8_t)label;
        for (int d = 0; d < 4; ++d) {
            a.box[k * 8 + 2 * d] = d < D ? lo[d] : 0.0;
            a.box[k * 8 + 2 * d + 1] = d < D ? hi[d] : 0.0;
        }
        a.depth[k] = (uint8_t)depth;
    }
}

// Gathers records through a permutation (shuffling the training set).
__global__ void k_gather(const bf16* __restrict__ fin, const uint8_t* __restrict__ cin, const int8_t* __restrict__ ain,
                         const unsigned* __restrict__ perm, size_t n, bf16* __restrict__ fout, uint8_t* __restrict__ cout,
                         int8_t* __restrict__ aout) {
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
        const size_t s = perm[r];
        for (int k = 0; k < NK; ++k) fout[r * NK + k] = fin[s * NK + k];
        cout[r] = cin[s];
        aout[r] = ain[s];
    }
}

// ------------------------------------------------------------------ host state
struct FamilyModel {
    float* master = nullptr;  // NPARAM
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    bf16* views = nullptr;    // NVIEW
    int* step = nullptr;
    float* loss = nullptr;
    bool ready = false;
};

struct ModelState {
    FamilyModel fam[6];
    // trace records (one family at a time)
    int rec_family = -1;
    size_t rec_cap = 0, rec_n = 0, rec_stride = 1, rec_phase = 0;
    bool collecting = false;
    bf16* rec_x = nullptr;
    uint8_t* rec_crit = nullptr;
    int8_t* rec_axis = nullptr;
    double* rec_box = nullptr;
    uint8_t* rec_depth = nullptr;
    unsigned long long* rec_count = nullptr;
    // inference kernel: 0 = warp-level mma.sync, 1 = tcgen05 with tensor memory
    // (default: the same forward pass the graph engine's level kernel runs inline,
    // so both engines take identical learned decisions)
    int infer_kind = 1;
    int* tc_err = nullptr;    // device flag raised by a timed-out tcgen05 wait
    int* tc_err_h = nullptr;  // pinned copy, refreshed after every tcgen05 launch
    int tc_wait_limit = kTcWaitLimit;
    // training kernel: 0 = warp-level mma.sync, 1 = tcgen05 (default)
    int train_kind = 1;
    // per-chunk hints
    uint8_t* hint_axis = nullptr;
    uint8_t* hint_order = nullptr;
    size_t hint_cap = 0;
};

cp_status ok_or(cudaError_t e) {
    if (e == cudaSuccess) return CP_OK;
    return cp_record_cuda_error(e, e == cudaErrorMemoryAllocation ? CP_ERR_NOMEM : CP_ERR_CUDA);
}
#define M_TRY(x)                    \
    do {                            \
        cp_status s_ = (x);         \
        if (s_ != CP_OK) return s_; \
    } while (0)

ModelState* state(cp_prover* p, bool create) {
    void*& slot = cp_prover_model(p);
    if (!slot && create) slot = new ModelState();
    return static_cast<ModelState*>(slot);
}

cp_status ensure_family(FamilyModel& f) {
    if (f.master) return CP_OK;
    M_TRY(ok_or(cudaMalloc(&f.master, sizeof(float) * NPARAM * 4)));
    f.m = f.master + NPARAM;
    f.v = f.m + NPARAM;
    f.grad = f.v + NPARAM;
    M_TRY(ok_or(cudaMalloc(&f.views, sizeof(bf16) * NVIEW)));
    M_TRY(ok_or(cudaMalloc(&f.step, sizeof(int) + sizeof(float))));
    f.loss = reinterpret_cast<float*>(f.step + 1);
    return CP_OK;
}

void free_family(FamilyModel& f) {
    cudaFree(f.master);
    cudaFree(f.views);
    cudaFree(f.step);
    f = FamilyModel();
}

void free_records(ModelState* m) {
    cudaFree(m->rec_x);
    cudaFree(m->rec_crit);
    cudaFree(m->rec_axis);
    cudaFree(m->rec_box);
    cudaFree(m->rec_depth);
    cudaFree(m->rec_count);
    m->rec_x = nullptr;
    m->rec_crit = nullptr;
    m->rec_axis = nullptr;
    m->rec_box = nullptr;
    m->rec_depth = nullptr;
    m->rec_count = nullptr;
    m->rec_cap = m->rec_n = 0;
    m->rec_family = -1;
}

// Deterministic initial parameters: uniform +-1/sqrt(fan_in) from a seeded
// 64-bit Mersenne twister; the padded input rows are zero.
std::vector<float> init_params(uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<float> p(NPARAM, 0.f);
    for (int i = 0; i < NPARAM; ++i) {
        const bool first = i < P_W2;
        const double scale = 1.0 / std::sqrt(first ? (double)NIN : (double)NH);
        const double x = u(rng) * scale;
        p[i] = (i < P_B1 && i >= NIN * NH) ? 0.f : (float)x;
    }
    return p;
}

size_t train_smem() { return sizeof(TrainSmem); }
size_t train_tc_smem() { return sizeof(TtSmem) + 1024; }  // + alignment of the tile base to 1024 B

// Training kernels: 0 = warp-level mma.sync (64 rows per block), 1 = tcgen05
// with tensor-memory accumulators (128 rows per CTA).  `err` (kind 1): device
// flag raised by a timed-out completion wait.
cp_status launch_train(const FamilyModel& f, const bf16* feats, const uint8_t* crit, const int8_t* axis, size_t n,
                       size_t row0, size_t rows, int fam, cudaStream_t st, bool with_step, int kind = 0,
                       int* err = nullptr, int wait_limit = kTcWaitLimit) {
    // per-device function attribute: set on every call (cheap), so a handle on
    // another device gets it too
    cudaError_t e = kind ? cudaFuncSetAttribute(k_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)train_tc_smem())
                         : cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)train_smem());
    if (e != cudaSuccess) return cp_record_cuda_error(e, CP_ERR_CUDA);
    TrainArgs a;
    a.feats = feats;
    a.crit = crit;
    a.axis = axis;
    a.row0 = row0;
    a.rows = rows;
    a.n = n;
    a.K = std::min(cp_family_criteria(fam), 4);
    a.D = family_dims(fam);
    a.inv_batch = 1.0f / (float)rows;
    a.views = f.views;
    a.master = f.master;
    a.grad = f.grad;
    a.loss = f.loss;
    a.step = with_step ? f.step : nullptr;
    if (kind) {
        if (!err) return cp_fail(CP_ERR_INVALID, "tcgen05 training needs an error flag");
        TtArgs t{a, err, wait_limit};
        const unsigned grid = (unsigned)((rows + kTcRows - 1) / kTcRows);
        k_train_tc<<<grid, kTcRows, train_tc_smem(), st>>>(t);
        return cp_check_launch();
    }
    const unsigned grid = (unsigned)((rows + kTrainRows - 1) / kTrainRows);
    k_train_step<<<grid, kTrainWarps * 32, train_smem(), st>>>(a);
    return cp_check_launch();
}

template <int FAM>
cp_status launch_infer_t(const InferArgs& a, cudaStream_t st) {
    const size_t groups = (a.count + kRowsPerWarp - 1) / kRowsPerWarp;
    unsigned grid = (unsigned)std::min<size_t>((groups + 3) / 4, 148 * 8);
    if (grid == 0) grid = 1;
    k_infer<FAM><<<grid, 128, 0, st>>>(a);
    return cp_check_launch();
}
cp_status launch_infer(int fam, const InferArgs& a, cudaStream_t st) {
    switch (fam) {
    case 0: return launch_infer_t<0>(a, st);
    case 1: return launch_infer_t<1>(a, st);
    case 2: return launch_infer_t<2>(a, st);
    case 3: return launch_infer_t<3>(a, st);
    case 4: return launch_infer_t<4>(a, st);
    default: return launch_infer_t<5>(a, st);
    }
}

template <int FAM>
cp_status launch_infer_tc_t(const TcArgs& a, cudaStream_t st) {
    const size_t tiles = (a.a.count + kTcRows - 1) / kTcRows;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(tiles, 148 * 4));
    // about 30 KB of static shared memory per CTA: the largest carveout lets the
    // four CTAs per SM that the tensor memory allows (128 columns each) be resident
    cudaFuncSetAttribute(k_infer_tc<FAM>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    k_infer_tc<FAM><<<grid, kTcRows, 0, st>>>(a);
    return cp_check_launch();
}
cp_status launch_infer_tc(int fam, const TcArgs& a, cudaStream_t st) {
    switch (fam) {
    case 0: return launch_infer_tc_t<0>(a, st);
    case 1: return launch_infer_tc_t<1>(a, st);
    case 2: return launch_infer_tc_t<2>(a, st);
    case 3: return launch_infer_tc_t<3>(a, st);
    case 4: return launch_infer_tc_t<4>(a, st);
    default: return launch_infer_tc_t<5>(a, st);
    }
}

template <int FAM>
cp_status launch_label_t(const LabelArgs& a, cudaStream_t st) {
    k_label<FAM><<<148 * 4, 128, 0, st>>>(a);
    return cp_check_launch();
}
cp_status launch_label(int fam, const LabelArgs& a, cudaStream_t st) {
    switch (fam) {
    case 0: return launch_label_t<0>(a, st);
    case 1: return launch_label_t<1>(a, st);
    case 2: return launch_label_t<2>(a, st);
    case 3: return launch_label_t<3>(a, st);
    case 4: return launch_label_t<4>(a, st);
    default: return launch_label_t<5>(a, st);
    }
}

}  // namespace

// Runs the configured inference kernel; with tcgen05, the device error flag of
// the previous launch is checked first and this launch's flag is copied to
// pinned memory behind it (the engine synchronises the stream between chunks).
cp_status run_infer(ModelState* m, int fam, const InferArgs& a, cudaStream_t st) {
    if (m->infer_kind == 0) return launch_infer(fam, a, st);
    if (!m->tc_err) {
        M_TRY(ok_or(cudaMalloc(&m->tc_err, sizeof(int))));
        M_TRY(ok_or(cudaMallocHost(&m->tc_err_h, sizeof(int))));
        *m->tc_err_h = 0;
        M_TRY(ok_or(cudaMemsetAsync(m->tc_err, 0, sizeof(int), st)));
    }
    if (*m->tc_err_h) return cp_fail(CP_ERR_DEVICE, "tcgen05 inference: a tensor-core completion wait timed out");
    TcArgs t;
    t.a = a;
    t.err = m->tc_err;
    t.wait_limit = m->tc_wait_limit;
    M_TRY(launch_infer_tc(fam, t, st));
    return ok_or(cudaMemcpyAsync(m->tc_err_h, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
}

// ------------------------------------------------------------------ engine hooks
cp_status cp_model_hints(cp_prover* p, int fam, const BoxList& in, size_t begin, size_t count, uint8_t** axis,
                         uint8_t** order) {
    ModelState* m = state(p, false);
    if (!m || !m->fam[fam].ready)
        return cp_fail(CP_ERR_INVALID, "no proposal model for family %d: train one (cp_model_train) or load "
                                       "parameters (cp_model_set_params)", fam);
    if (m->hint_cap < count) {
        cudaFree(m->hint_axis);
        m->hint_axis = nullptr;
        m->hint_cap = 0;
        M_TRY(ok_or(cudaMalloc(&m->hint_axis, 2 * count)));
        m->hint_order = m->hint_axis + count;
        m->hint_cap = count;
    }
    InferArgs a;
    a.in = in;
    a.begin = begin;
    a.count = count;
    a.views = m->fam[fam].views;
    a.master = m->fam[fam].master;
    a.axis = axis ? m->hint_axis : nullptr;
    a.order = order ? m->hint_order : nullptr;
    a.logits = nullptr;
    M_TRY(run_infer(m, fam, a, cp_prover_stream(p)));
    if (axis) *axis = m->hint_axis;
    if (order) *order = m->hint_order;
    return CP_OK;
}

cp_status cp_model_net_params(cp_prover* p, int fam, const void** views, const float** master, int* wait_limit) {
    ModelState* m = state(p, false);
    if (!m || fam < 0 || fam > 5 || !m->fam[fam].ready)
        return cp_fail(CP_ERR_INVALID, "no proposal model for family %d: train one (cp_model_train) or load "
                                       "parameters (cp_model_set_params)", fam);
    *views = m->fam[fam].views;
    *master = m->fam[fam].master;
    *wait_limit = m->tc_wait_limit;
    return CP_OK;
}

cp_status cp_model_collect_chunk(cp_prover* p, int fam, const BoxList& in, size_t begin, size_t count,
                                 const double* tab_t, const double* tab_v, int tab_n, double tab_h) {
    ModelState* m = state(p, false);
    if (!m || !m->collecting || m->rec_family != fam || count == 0) return CP_OK;
    LabelArgs a;
    a.in = in;
    a.begin = begin;
    a.count = count;
    a.stride = m->rec_stride;
    a.phase = m->rec_phase % m->rec_stride;
    m->rec_phase += 7919;  // vary the sampled residue between chunks
    a.tab = SingleTable{tab_t, tab_v, tab_n, tab_h};
    a.feats = m->rec_x;
    a.crit = m->rec_crit;
    a.axis = m->rec_axis;
    a.box = m->rec_box;
    a.depth = m->rec_depth;
    a.count_out = m->rec_count;
    a.cap = m->rec_cap;
    return launch_label(fam, a, cp_prover_stream(p));
}

bool cp_model_collecting(cp_prover* p) {
    ModelState* m = state(p, false);
    return m && m->collecting;
}

void cp_model_free(cp_prover* p) {
    ModelState* m = state(p, false);
    if (!m) return;
    for (auto& f : m->fam) free_family(f);
    free_records(m);
    cudaFree(m->hint_axis);
    cudaFree(m->tc_err);
    cudaFreeHost(m->tc_err_h);
    delete m;
    cp_prover_model(p) = nullptr;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

cp_status cp_model_collect(cp_prover* p, const cp_refine_opts* o, int64_t max_records, int32_t sample_stride,
                           int64_t* n_records) {
    if (!p || !o || max_records <= 0 || sample_stride <= 0 || o->family < 0 || o->family > 5)
        return cp_fail(CP_ERR_INVALID, "cp_model_collect: invalid arguments");
    if (o->policy == CP_SPLIT_LEARNED || o->learned_order)
        return cp_fail(CP_ERR_INVALID, "cp_model_collect: record with a plain policy (the model is being built)");
    ModelState* m = state(p, true);
    if (m->rec_cap != (size_t)max_records) {
        free_records(m);
        const size_t cap = (size_t)max_records;
        M_TRY(ok_or(cudaMalloc(&m->rec_x, sizeof(bf16) * NK * cap)));
        M_TRY(ok_or(cudaMalloc(&m->rec_crit, cap)));
        M_TRY(ok_or(cudaMalloc(&m->rec_axis, cap)));
        M_TRY(ok_or(cudaMalloc(&m->rec_box, sizeof(double) * 8 * cap)));
        M_TRY(ok_or(cudaMalloc(&m->rec_depth, cap)));
        M_TRY(ok_or(cudaMalloc(&m->rec_count, sizeof(unsigned long long))));
        m->rec_cap = cap;
    }
    cudaStream_t st = cp_prover_stream(p);
    M_TRY(ok_or(cudaMemsetAsync(m->rec_count, 0, sizeof(unsigned long long), st)));
    m->rec_family = o->family;
    m->rec_stride = (size_t)sample_stride;
    m->rec_phase = 0;
    m->collecting = true;
    cp_refine_report r;
    cp_status s = cp_refine(p, o, &r);
    m->collecting = false;
    if (s != CP_OK) return s;
    unsigned long long n = 0;
    M_TRY(ok_or(cudaMemcpyAsync(&n, m->rec_count, sizeof(n), cudaMemcpyDeviceToHost, st)));
    M_TRY(ok_or(cudaStreamSynchronize(st)));
    m->rec_n = (size_t)std::min<unsigned long long>(n, m->rec_cap);
    if (n_records) *n_records = (int64_t)m->rec_n;
    return CP_OK;
}

cp_status cp_model_records(cp_prover* p, float* feats, uint8_t* crit, int8_t* axis, double* boxes, uint8_t* depth,
                           size_t cap, size_t* n) {
    ModelState* m = state(p, false);
    if (!m || !n) return cp_fail(CP_ERR_INVALID, "cp_model_records: no records");
    const size_t k = std::min(cap, m->rec_n);
    *n = m->rec_n;
    if (k == 0) return CP_OK;
    cudaStream_t st = cp_prover_stream(p);
    if (feats) {
        std::vector<bf16> tmp(k * NK);
        M_TRY(ok_or(cudaMemcpyAsync(tmp.data(), m->rec_x, sizeof(bf16) * NK * k, cudaMemcpyDeviceToHost, st)));
        M_TRY(ok_or(cudaStreamSynchronize(st)));
        for (size_t i = 0; i < k * NK; ++i) feats[i] = __bfloat162float(tmp[i]);
    }
    if (crit) M_TRY(ok_or(cudaMemcpyAsync(crit, m->rec_crit, k, cudaMemcpyDeviceToHost, st)));
    if (axis) M_TRY(ok_or(cudaMemcpyAsync(axis, m->rec_axis, k, cudaMemcpyDeviceToHost, st)));
    if (boxes) M_TRY(ok_or(cudaMemcpyAsync(boxes, m->rec_box, sizeof(double) * 8 * k, cudaMemcpyDeviceToHost, st)));
    if (depth) M_TRY(ok_or(cudaMemcpyAsync(depth, m->rec_depth, k, cudaMemcpyDeviceToHost, st)));
    return ok_or(cudaStreamSynchronize(st));
}

cp_status cp_model_train(cp_prover* p, int family, int epochs, int batch, float lr, uint64_t seed, float* losses) {
    ModelState* m = state(p, false);
    if (!m || m->rec_family != family || m->rec_n == 0)
        return cp_fail(CP_ERR_INVALID, "cp_model_train: collect records of family %d first", family);
    if (epochs <= 0 || batch <= 0 || batch % kTrainRows != 0 || !(lr > 0.f))
        return cp_fail(CP_ERR_INVALID, "cp_model_train: epochs > 0, batch a positive multiple of %d, lr > 0",
                       kTrainRows);
    FamilyModel& f = m->fam[family];
    M_TRY(ensure_family(f));
    cudaStream_t st = cp_prover_stream(p);
    if (m->train_kind && !m->tc_err) {
        M_TRY(ok_or(cudaMalloc(&m->tc_err, sizeof(int))));
        M_TRY(ok_or(cudaMallocHost(&m->tc_err_h, sizeof(int))));
        *m->tc_err_h = 0;
        M_TRY(ok_or(cudaMemsetAsync(m->tc_err, 0, sizeof(int), st)));
    }
    if (m->train_kind && *m->tc_err_h)
        return cp_fail(CP_ERR_DEVICE, "tcgen05 kernels: a tensor-core completion wait timed out earlier");
    const std::vector<float> init = init_params(seed);
    M_TRY(ok_or(cudaMemcpyAsync(f.master, init.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice, st)));
    M_TRY(ok_or(cudaMemsetAsync(f.m, 0, sizeof(float) * NPARAM * 3, st)));
    M_TRY(ok_or(cudaMemsetAsync(f.step, 0, sizeof(int) + sizeof(float), st)));
    k_views<<<(NPARAM + 255) / 256, 256, 0, st>>>(f.master, f.views);
    M_TRY(cp_check_launch());
    // shuffle once (seeded), then iterate the shuffled set every epoch
    const size_t n = m->rec_n;
    std::vector<unsigned> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = (unsigned)i;
    std::mt19937_64 rng(seed ^ 0x9E3779B97F4A7C15ull);
    std::shuffle(perm.begin(), perm.end(), rng);
    unsigned* dperm = nullptr;
    bf16* sx = nullptr;
    uint8_t* sc = nullptr;
    M_TRY(ok_or(cudaMalloc(&dperm, sizeof(unsigned) * n)));
    cp_status s = ok_or(cudaMalloc(&sx, sizeof(bf16) * NK * n + 2 * n));
    if (s == CP_OK) {
        sc = reinterpret_cast<uint8_t*>(sx + NK * n);
        int8_t* sa = reinterpret_cast<int8_t*>(sc + n);
        s = ok_or(cudaMemcpyAsync(dperm, perm.data(), sizeof(unsigned) * n, cudaMemcpyHostToDevice, st));
        if (s == CP_OK) {
            k_gather<<<512, 256, 0, st>>>(m->rec_x, m->rec_crit, m->rec_axis, dperm, n, sx, sc, sa);
            s = cp_check_launch();
        }
        const size_t steps = std::max<size_t>(1, n / (size_t)batch);
        for (int e = 0; e < epochs && s == CP_OK; ++e) {
            s = ok_or(cudaMemsetAsync(f.loss, 0, sizeof(float), st));
            for (size_t b = 0; b < steps && s == CP_OK; ++b) {
                const size_t row0 = b * (size_t)batch;
                const size_t rows = std::min<size_t>((size_t)batch, n - row0);
                s = launch_train(f, sx, sc, sa, n, row0, rows, family, st, true, m->train_kind, m->tc_err,
                                 m->tc_wait_limit);
                if (s == CP_OK) {
                    k_adam<<<(NPARAM + 255) / 256, 256, 0, st>>>(f.master, f.m, f.v, f.grad, f.views, f.step, lr);
                    s = cp_check_launch();
                }
            }
            if (s == CP_OK && losses) {
                float l = 0.f;
                s = ok_or(cudaMemcpyAsync(&l, f.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
                if (s == CP_OK) s = ok_or(cudaStreamSynchronize(st));
                losses[e] = l / (float)steps;
            }
        }
        if (s == CP_OK) s = ok_or(cudaStreamSynchronize(st));
        if (s == CP_OK && m->train_kind) {
            s = ok_or(cudaMemcpy(m->tc_err_h, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
            if (s == CP_OK && *m->tc_err_h)
                s = cp_fail(CP_ERR_DEVICE, "tcgen05 training: a tensor-core completion wait timed out");
        }
    }
    cudaFree(dperm);
    cudaFree(sx);
    if (s == CP_OK) f.ready = true;
    return s;
}

cp_status cp_model_set_training(cp_prover* p, int kind) {
    if (!p || kind < 0 || kind > 1) return cp_fail(CP_ERR_INVALID, "cp_model_set_training: kind 0 or 1");
    state(p, true)->train_kind = kind;
    return CP_OK;
}

cp_status cp_model_get_params(cp_prover* p, int family, float* params) {
    ModelState* m = state(p, false);
    if (!m || family < 0 || family > 5 || !m->fam[family].ready || !params)
        return cp_fail(CP_ERR_INVALID, "cp_model_get_params: no model for family %d", family);
    cudaStream_t st = cp_prover_stream(p);
    M_TRY(ok_or(cudaMemcpyAsync(params, m->fam[family].master, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, st)));
    return ok_or(cudaStreamSynchronize(st));
}

cp_status cp_model_set_params(cp_prover* p, int family, const float* params) {
    if (!p || family < 0 || family > 5 || !params) return cp_fail(CP_ERR_INVALID, "cp_model_set_params: bad arguments");
    ModelState* m = state(p, true);
    FamilyModel& f = m->fam[family];
    M_TRY(ensure_family(f));
    cudaStream_t st = cp_prover_stream(p);
    M_TRY(ok_or(cudaMemcpyAsync(f.master, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, st)));
    M_TRY(ok_or(cudaMemsetAsync(f.m, 0, sizeof(float) * NPARAM * 3, st)));
    k_views<<<(NPARAM + 255) / 256, 256, 0, st>>>(f.master, f.views);
    M_TRY(cp_check_launch());
    M_TRY(ok_or(cudaStreamSynchronize(st)));
    f.ready = true;
    return CP_OK;
}

int cp_model_param_count(void) { return NPARAM; }

// One forward + backward pass on the GPU over host rows (no optimiser step);
// for gradient checks.  feats: [n][16] FP32 (rounded to BF16 on the device).
cp_status cp_model_loss_grad(int family, const float* params, const float* feats, const uint8_t* crit,
                             const int8_t* axis, size_t n, float* loss, float* grad) {
    return cp_model_loss_grad_kind(0, family, params, feats, crit, axis, n, loss, grad);
}

cp_status cp_model_loss_grad_kind(int kind, int family, const float* params, const float* feats, const uint8_t* crit,
                                  const int8_t* axis, size_t n, float* loss, float* grad) {
    if (kind < 0 || kind > 1 || family < 0 || family > 5 || !params || !feats || !crit || !axis || n == 0 || !loss ||
        !grad)
        return cp_fail(CP_ERR_INVALID, "cp_model_loss_grad: bad arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return cp_fail(CP_ERR_NO_DEVICE, "no CUDA device");
    }
    FamilyModel f;
    cp_status s = ensure_family(f);
    bf16* dx = nullptr;
    int* derr = nullptr;
    if (s == CP_OK) s = ok_or(cudaMalloc(&dx, sizeof(bf16) * NK * n + 2 * n));
    if (s == CP_OK) s = ok_or(cudaMalloc(&derr, sizeof(int)));
    if (s == CP_OK) s = ok_or(cudaMemset(derr, 0, sizeof(int)));
    if (s == CP_OK) {
        std::vector<bf16> hx(NK * n);
        for (size_t i = 0; i < NK * n; ++i) hx[i] = __float2bfloat16_rn(feats[i]);
        uint8_t* dc = reinterpret_cast<uint8_t*>(dx + NK * n);
        int8_t* da = reinterpret_cast<int8_t*>(dc + n);
        s = ok_or(cudaMemcpy(dx, hx.data(), sizeof(bf16) * NK * n, cudaMemcpyHostToDevice));
        if (s == CP_OK) s = ok_or(cudaMemcpy(dc, crit, n, cudaMemcpyHostToDevice));
        if (s == CP_OK) s = ok_or(cudaMemcpy(da, axis, n, cudaMemcpyHostToDevice));
        if (s == CP_OK) s = ok_or(cudaMemcpy(f.master, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
        if (s == CP_OK) s = ok_or(cudaMemset(f.grad, 0, sizeof(float) * NPARAM));
        if (s == CP_OK) s = ok_or(cudaMemset(f.loss, 0, sizeof(float)));
        if (s == CP_OK) {
            k_views<<<(NPARAM + 255) / 256, 256>>>(f.master, f.views);
            s = cp_check_launch();
        }
        if (s == CP_OK) s = launch_train(f, dx, dc, da, n, 0, n, family, 0, false, kind, derr);
        if (s == CP_OK) s = ok_or(cudaDeviceSynchronize());
        int herr = 0;
        if (s == CP_OK) s = ok_or(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
        if (s == CP_OK && herr) s = cp_fail(CP_ERR_DEVICE, "tcgen05 training: a tensor-core completion wait timed out");
        if (s == CP_OK) s = ok_or(cudaMemcpy(grad, f.grad, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
        if (s == CP_OK) s = ok_or(cudaMemcpy(loss, f.loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    cudaFree(dx);
    cudaFree(derr);
    free_family(f);
    return s;
}

// Network outputs and decisions for host boxes (lo/hi SoA with stride n).
cp_status cp_model_predict(cp_prover* p, int family, const double* lo, const double* hi, const uint8_t* depth,
                           size_t n, float* logits, uint8_t* axis, uint8_t* order) {
    ModelState* m = state(p, false);
    if (!m || family < 0 || family > 5 || !m->fam[family].ready || !lo || !hi || n == 0)
        return cp_fail(CP_ERR_INVALID, "cp_model_predict: no model for family %d or bad arguments", family);
    const int D = family_dims(family);
    cudaStream_t st = cp_prover_stream(p);
    double* dlo = nullptr;
    cp_status s = ok_or(cudaMalloc(&dlo, sizeof(double) * 2 * D * n + n + 2 * n + sizeof(float) * NO * n + 16));
    if (s == CP_OK) {
        double* dhi = dlo + D * n;
        uint8_t* dd = reinterpret_cast<uint8_t*>(dhi + D * n);
        uint8_t* dax = dd + n;
        uint8_t* dor = dax + n;
        float* dlg = reinterpret_cast<float*>(((uintptr_t)(dor + n) + 15) & ~(uintptr_t)15);
        s = ok_or(cudaMemcpyAsync(dlo, lo, sizeof(double) * D * n, cudaMemcpyHostToDevice, st));
        if (s == CP_OK) s = ok_or(cudaMemcpyAsync(dhi, hi, sizeof(double) * D * n, cudaMemcpyHostToDevice, st));
        if (s == CP_OK)
            s = depth ? ok_or(cudaMemcpyAsync(dd, depth, n, cudaMemcpyHostToDevice, st))
                      : ok_or(cudaMemsetAsync(dd, 0, n, st));
        if (s == CP_OK) {
            InferArgs a;
            a.in = BoxList{dlo, dhi, dd, n};
            a.begin = 0;
            a.count = n;
            a.views = m->fam[family].views;
            a.master = m->fam[family].master;
            a.axis = dax;
            a.order = dor;
            a.logits = dlg;
            s = run_infer(m, family, a, st);
        }
        if (s == CP_OK && logits)
            s = ok_or(cudaMemcpyAsync(logits, dlg, sizeof(float) * NO * n, cudaMemcpyDeviceToHost, st));
        if (s == CP_OK && axis) s = ok_or(cudaMemcpyAsync(axis, dax, n, cudaMemcpyDeviceToHost, st));
        if (s == CP_OK && order) s = ok_or(cudaMemcpyAsync(order, dor, n, cudaMemcpyDeviceToHost, st));
        if (s == CP_OK) s = ok_or(cudaStreamSynchronize(st));
        if (s == CP_OK && m->infer_kind && m->tc_err_h && *m->tc_err_h)
            s = cp_fail(CP_ERR_DEVICE, "tcgen05 inference: a tensor-core completion wait timed out");
    }
    cudaFree(dlo);
    return s;
}

cp_status cp_model_set_inference(cp_prover* p, int kind) {
    if (!p || kind < 0 || kind > 1) return cp_fail(CP_ERR_INVALID, "cp_model_set_inference: kind 0 or 1");
    ModelState* m = state(p, true);
    m->infer_kind = kind;
    // a time-out recorded by an earlier tcgen05 launch is cleared
    if (m->tc_err) {
        cudaStream_t st = cp_prover_stream(p);
        M_TRY(ok_or(cudaStreamSynchronize(st)));
        M_TRY(ok_or(cudaMemsetAsync(m->tc_err, 0, sizeof(int), st)));
        M_TRY(ok_or(cudaStreamSynchronize(st)));
        *m->tc_err_h = 0;
    }
    return CP_OK;
}

cp_status cp_model_set_wait_limit(cp_prover* p, int32_t polls) {
    if (!p || polls < 0) return cp_fail(CP_ERR_INVALID, "cp_model_set_wait_limit: polls >= 0");
    state(p, true)->tc_wait_limit = polls;
    return CP_OK;
}

}  // extern "C"
