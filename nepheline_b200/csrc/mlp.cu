// SPDX-License-Identifier: Apache-2.0
//
// The learned warm start's network on the tensor cores: a 16 -> 64 -> 64 -> 64 -> 3
// perceptron with ReLU, BF16 weights and activations, FP32 accumulation (the reference has no
// counterpart: its new contact points start at zero impulse, contact.c:547-565).
//
// A warp owns a tile of 16 samples. Each layer is mma.sync m16n8k16 (bf16 x bf16 -> f32): the
// tile's activations are the A fragments, the weights (staged once per block in shared
// memory, row-major [out][in], and transposed for the backward pass) the B fragments. A
// layer's accumulators become the next layer's A fragments in registers: the accumulator of
// columns (2t, 2t+1) of rows g and g+8 is exactly what the A fragment needs, so only a bias,
// a ReLU and a conversion to bf16 sit between layers. The network is 64 units wide: a
// 16-sample warp tile keeps a whole forward and backward pass in registers, which a
// 128-row tcgen05 tile with its TMEM round trips would not improve at this width (measured, the
// forward kernel is bound by instruction issue and the gradient kernel by its shared-memory
// adds of the weight gradients, neither by the tensor pipe).
//
// Training: mean squared error on the three outputs; the backward pass propagates through
// the same fragments (dH = dZ W on the tensor cores with the transposed weights), and the
// weight gradients dW = dZ^T H are 16-sample tensor-core products accumulated per block in
// shared memory, then once per block in global memory. Adam updates FP32 master weights and
// refreshes their BF16 copies.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "nepheline_b200.h"

namespace {

constexpr int kIn = NPH_GPU_MLP_INPUTS;    // 16
constexpr int kHid = NPH_GPU_MLP_HIDDEN;   // 64
constexpr int kOut = NPH_GPU_MLP_OUTPUTS;  // 3
constexpr int kOutPad = 8;                 // one mma n-tile

// Parameter offsets in the FP32 master vector (row-major [out][in] weights, then biases).
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kHid * kIn;
constexpr int kW2 = kB1 + kHid;
constexpr int kB2 = kW2 + kHid * kHid;
constexpr int kW3 = kB2 + kHid;
constexpr int kB3 = kW3 + kHid * kHid;
constexpr int kW4 = kB3 + kHid;
constexpr int kB4 = kW4 + kOut * kHid;
constexpr int kParams = kB4 + kOut;
static_assert(kParams == NPH_GPU_MLP_PARAMS, "parameter count");

constexpr int kWarps = 4;            // per block
constexpr int kThreads = 32 * kWarps;
constexpr int kTile = 16;            // samples per warp tile
// Shared-memory rows are padded by 8 bf16 (16 bytes): a fragment's eight rows then start in
// eight different groups of four banks, so a warp's 32 fragment loads hit 32 banks (unpadded,
// rows of 64 bf16 are 32 words apart and eight lanes share each bank).
constexpr int kPad = 8;
constexpr int kInRow = kIn + kPad;
constexpr int kHidRow = kHid + kPad;

// Shared memory of a block: the bf16 weights (and transposes), fp32 biases.
struct SmemWeights {
    __nv_bfloat16 w1[kHid][kInRow];      // [out][in]
    __nv_bfloat16 w2[kHid][kHidRow];
    __nv_bfloat16 w3[kHid][kHidRow];
    __nv_bfloat16 w4[kOutPad][kHidRow];  // rows >= 3 zero
    __nv_bfloat16 w2t[kHid][kHidRow];    // [in][out]
    __nv_bfloat16 w3t[kHid][kHidRow];
    __nv_bfloat16 w4t[kHid][16 + kPad];  // [in][out], out padded to one k-step
    float b1[kHid], b2[kHid], b3[kHid], b4[kOutPad];
};

// A warp's scratch for the backward pass: a layer's dZ and input, bf16, [sample][unit].
struct SmemTile {
    __nv_bfloat16 dz[kTile][kHidRow];
    __nv_bfloat16 h[kTile][kHidRow];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t pair(const __nv_bfloat16 *p)
{
    return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ uint32_t pair2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    __nv_bfloat162 v;
    v.x = lo;
    v.y = hi;
    return *reinterpret_cast<const uint32_t *>(&v);
}

// D (16x8 f32) += A (16x16 bf16, row) * B (16x8 bf16, col).
__device__ __forceinline__ void mma(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of rows [16 kt, 16 kt + 16) (the k index) and columns [8 nt, 8 nt + 8) (the n
// index) of a matrix stored [n][k] (row-major by n), rows K bf16 apart.
template <int K>
__device__ __forceinline__ void b_frag(const __nv_bfloat16 (*w)[K], int nt, int kt, int g, int t,
                                       uint32_t &b0, uint32_t &b1)
{
    b0 = pair(&w[nt * 8 + g][kt * 16 + 2 * t]);
    b1 = pair(&w[nt * 8 + g][kt * 16 + 2 * t + 8]);
}

// Accumulators of 8 n-tiles (64 columns) to A fragments of 4 k-steps, with bias and ReLU.
__device__ __forceinline__ void relu_to_a(float d[8][4], const float *bias, int t, uint32_t a[4][4],
                                          bool mask[8][4])
{
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * t;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float z = d[nt][i] + bias[c + (i & 1)];
            mask[nt][i] = z > 0.0f;
            d[nt][i] = z > 0.0f ? z : 0.0f;
        }
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        a[kt][0] = pack_bf16(d[2 * kt][0], d[2 * kt][1]);
        a[kt][1] = pack_bf16(d[2 * kt][2], d[2 * kt][3]);
        a[kt][2] = pack_bf16(d[2 * kt + 1][0], d[2 * kt + 1][1]);
        a[kt][3] = pack_bf16(d[2 * kt + 1][2], d[2 * kt + 1][3]);
    }
}

// The input tile's A fragments: 16 samples x 16 features (fp32 in global memory, row-major).
__device__ __forceinline__ void input_frag(const float *x, uint32_t count, uint32_t row0, int g,
                                           int t, uint32_t a[4])
{
    auto at = [&](int r, int c) -> float {
        const uint32_t row = row0 + (uint32_t)r;
        return row < count ? x[(size_t)row * kIn + c] : 0.0f;
    };
    a[0] = pack_bf16(at(g, 2 * t), at(g, 2 * t + 1));
    a[1] = pack_bf16(at(g + 8, 2 * t), at(g + 8, 2 * t + 1));
    a[2] = pack_bf16(at(g, 2 * t + 8), at(g, 2 * t + 9));
    a[3] = pack_bf16(at(g + 8, 2 * t + 8), at(g + 8, 2 * t + 9));
}

struct Forward {
    uint32_t a0[4];      // input
    uint32_t a1[4][4];   // h1 (bf16, post-ReLU)
    uint32_t a2[4][4];   // h2
    uint32_t a3[4][4];   // h3
    bool m1[8][4], m2[8][4], m3[8][4];
    float y[4];          // outputs: cols 2t, 2t+1 of rows g, g+8 (cols < 3 valid)
};

__device__ __forceinline__ void forward(const SmemWeights &W, const float *x, uint32_t count,
                                        uint32_t row0, int g, int t, Forward &F)
{
    input_frag(x, count, row0, g, t, F.a0);
    float d[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0f;
        uint32_t b0, b1;
        b_frag<kInRow>(W.w1, nt, 0, g, t, b0, b1);
        mma(d[nt], F.a0, b0, b1);
    }
    relu_to_a(d, W.b1, t, F.a1, F.m1);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            uint32_t b0, b1;
            b_frag<kHidRow>(W.w2, nt, kt, g, t, b0, b1);
            mma(d[nt], F.a1[kt], b0, b1);
        }
    }
    relu_to_a(d, W.b2, t, F.a2, F.m2);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            uint32_t b0, b1;
            b_frag<kHidRow>(W.w3, nt, kt, g, t, b0, b1);
            mma(d[nt], F.a2[kt], b0, b1);
        }
    }
    relu_to_a(d, W.b3, t, F.a3, F.m3);
    F.y[0] = F.y[1] = F.y[2] = F.y[3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        uint32_t b0, b1;
        b_frag<kHidRow>(W.w4, 0, kt, g, t, b0, b1);
        mma(F.y, F.a3[kt], b0, b1);
    }
    const int c = 2 * t;
    F.y[0] += W.b4[c];
    F.y[1] += W.b4[c + 1];
    F.y[2] += W.b4[c];
    F.y[3] += W.b4[c + 1];
}

__device__ void load_weights(SmemWeights &W, const __nv_bfloat16 *wb, const float *master)
{
    for (int i = threadIdx.x; i < kHid * kIn; i += blockDim.x) {
        W.w1[i / kIn][i % kIn] = wb[kW1 + i];
    }
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int o = i / kHid, k = i % kHid;
        W.w2[o][k] = wb[kW2 + i];
        W.w3[o][k] = wb[kW3 + i];
        W.w2t[k][o] = wb[kW2 + i];
        W.w3t[k][o] = wb[kW3 + i];
    }
    for (int i = threadIdx.x; i < kOutPad * kHid; i += blockDim.x) {
        const int o = i / kHid, k = i % kHid;
        W.w4[o][k] = o < kOut ? wb[kW4 + o * kHid + k] : __float2bfloat16(0.0f);
    }
    for (int i = threadIdx.x; i < kHid * 16; i += blockDim.x) {
        const int k = i / 16, o = i % 16;
        W.w4t[k][o] = o < kOut ? wb[kW4 + o * kHid + k] : __float2bfloat16(0.0f);
    }
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        W.b1[i] = master[kB1 + i];
        W.b2[i] = master[kB2 + i];
        W.b3[i] = master[kB3 + i];
    }
    for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) {
        W.b4[i] = i < kOut ? master[kB4 + i] : 0.0f;
    }
    __syncthreads();
}

// Inference: y = f(x) for `count` samples (rows of 16 features; the first *count_dev of them
// when count_dev is given), written as rows of 3.
__global__ void __launch_bounds__(kThreads) k_mlp_forward(const float *x, uint32_t count,
                                                          const uint32_t *count_dev,
                                                          const __nv_bfloat16 *wb, const float *master,
                                                          float *y)
{
    __shared__ SmemWeights W;
    if (count_dev != nullptr) {
        count = min(count, *count_dev);
    }
    load_weights(W, wb, master);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles; tile += gridDim.x * kWarps) {
        const uint32_t row0 = tile * kTile;
        Forward F;
        forward(W, x, count, row0, g, t, F);
        const int c = 2 * t;
        const uint32_t r0 = row0 + g, r1 = row0 + g + 8;
        if (c < kOut) {
            if (r0 < count) {
                y[(size_t)r0 * kOut + c] = F.y[0];
            }
            if (r1 < count) {
                y[(size_t)r1 * kOut + c] = F.y[2];
            }
        }
        if (c + 1 < kOut) {
            if (r0 < count) {
                y[(size_t)r0 * kOut + c + 1] = F.y[1];
            }
            if (r1 < count) {
                y[(size_t)r1 * kOut + c + 1] = F.y[3];
            }
        }
    }
}

// dZ (accumulators of 8 n-tiles) to shared memory as bf16 [sample][unit].
__device__ __forceinline__ void store_tile(__nv_bfloat16 (*dst)[kHidRow], const float d[8][4], int g, int t)
{
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * t;
        dst[g][c] = __float2bfloat16(d[nt][0]);
        dst[g][c + 1] = __float2bfloat16(d[nt][1]);
        dst[g + 8][c] = __float2bfloat16(d[nt][2]);
        dst[g + 8][c + 1] = __float2bfloat16(d[nt][3]);
    }
}

// An A-fragment set (4 k-steps, 16 samples x 64 units) to shared memory [sample][unit].
__device__ __forceinline__ void store_a(__nv_bfloat16 (*dst)[kHidRow], const uint32_t a[4][4], int g, int t)
{
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        const int c = kt * 16 + 2 * t;
        *reinterpret_cast<uint32_t *>(&dst[g][c]) = a[kt][0];
        *reinterpret_cast<uint32_t *>(&dst[g + 8][c]) = a[kt][1];
        *reinterpret_cast<uint32_t *>(&dst[g][c + 8]) = a[kt][2];
        *reinterpret_cast<uint32_t *>(&dst[g + 8][c + 8]) = a[kt][3];
    }
}

// The block's FP32 gradient in shared memory: each weight matrix's rows kAccPad floats longer
// than the matrix is wide, so that a warp's 32 atomic adds of one tensor-core tile (eight rows,
// four column pairs) fall in distinct banks but for pairs (the rows 64 floats apart put them in
// four banks), then the biases.
constexpr int kAccPad = 4;
constexpr int kAccW1 = 0;
constexpr int kAccW2 = kAccW1 + kHid * (kIn + kAccPad);
constexpr int kAccW3 = kAccW2 + kHid * (kHid + kAccPad);
constexpr int kAccW4 = kAccW3 + kHid * (kHid + kAccPad);
constexpr int kAccB1 = kAccW4 + kOut * (kHid + kAccPad);
constexpr int kAccB2 = kAccB1 + kHid;
constexpr int kAccB3 = kAccB2 + kHid;
constexpr int kAccB4 = kAccB3 + kHid;
constexpr int kAcc = kAccB4 + kOut;

// The accumulator slot of parameter p.
__device__ __forceinline__ int acc_index(int p)
{
    if (p < kB1) {
        return kAccW1 + (p - kW1) / kIn * (kIn + kAccPad) + (p - kW1) % kIn;
    }
    if (p < kW2) {
        return kAccB1 + p - kB1;
    }
    if (p < kB2) {
        return kAccW2 + (p - kW2) / kHid * (kHid + kAccPad) + (p - kW2) % kHid;
    }
    if (p < kW3) {
        return kAccB2 + p - kB2;
    }
    if (p < kB3) {
        return kAccW3 + (p - kW3) / kHid * (kHid + kAccPad) + (p - kW3) % kHid;
    }
    if (p < kW4) {
        return kAccB3 + p - kB3;
    }
    if (p < kB4) {
        return kAccW4 + (p - kW4) / kHid * (kHid + kAccPad) + (p - kW4) % kHid;
    }
    return kAccB4 + p - kB4;
}

// grad[o][i] += sum over the tile's 16 samples of dz[s][o] h[s][i], for O outputs x I inputs,
// on the tensor cores (A = dz^T, B = h), accumulated into fp32 shared memory (rows I + kAccPad
// floats apart).
template <int O, int I>
__device__ void weight_grad(const __nv_bfloat16 (*dz)[kHidRow], const __nv_bfloat16 (*h)[kHidRow], float *grad,
                            int g, int t)
{
    for (int mt = 0; mt < (O + 15) / 16; ++mt) {
        uint32_t a[4];
        auto dzv = [&](int s, int o) -> __nv_bfloat16 {
            return o < O ? dz[s][o] : __float2bfloat16(0.0f);
        };
        const int o0 = mt * 16 + g, o1 = mt * 16 + g + 8;
        a[0] = pair2(dzv(2 * t, o0), dzv(2 * t + 1, o0));
        a[1] = pair2(dzv(2 * t, o1), dzv(2 * t + 1, o1));
        a[2] = pair2(dzv(2 * t + 8, o0), dzv(2 * t + 9, o0));
        a[3] = pair2(dzv(2 * t + 8, o1), dzv(2 * t + 9, o1));
#pragma unroll
        for (int nt = 0; nt < I / 8; ++nt) {
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            const int i = nt * 8 + g;
            const uint32_t b0 = pair2(h[2 * t][i], h[2 * t + 1][i]);
            const uint32_t b1 = pair2(h[2 * t + 8][i], h[2 * t + 9][i]);
            mma(d, a, b0, b1);
            const int c = nt * 8 + 2 * t;
            constexpr int kRow = I + kAccPad;
            if (o0 < O) {
                atomicAdd(&grad[o0 * kRow + c], d[0]);
                atomicAdd(&grad[o0 * kRow + c + 1], d[1]);
            }
            if (o1 < O) {
                atomicAdd(&grad[o1 * kRow + c], d[2]);
                atomicAdd(&grad[o1 * kRow + c + 1], d[3]);
            }
        }
    }
}

// dH = dZ W: dz fragments (A, 4 k-steps over the layer's outputs) times the transposed weights.
__device__ __forceinline__ void back_mm(const uint32_t dz[4][4], const __nv_bfloat16 (*wt)[kHidRow], int g,
                                        int t, float d[8][4])
{
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            uint32_t b0, b1;
            b_frag<kHidRow>(wt, nt, kt, g, t, b0, b1);
            mma(d[nt], dz[kt], b0, b1);
        }
    }
}

__device__ __forceinline__ void mask_to_a(float d[8][4], const bool m[8][4], uint32_t a[4][4])
{
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            d[nt][i] = m[nt][i] ? d[nt][i] : 0.0f;
        }
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        a[kt][0] = pack_bf16(d[2 * kt][0], d[2 * kt][1]);
        a[kt][1] = pack_bf16(d[2 * kt][2], d[2 * kt][3]);
        a[kt][2] = pack_bf16(d[2 * kt + 1][0], d[2 * kt + 1][1]);
        a[kt][3] = pack_bf16(d[2 * kt + 1][2], d[2 * kt + 1][3]);
    }
}

// A gradient block's shared memory (dynamic: above the 48 KiB static limit).
struct GradSmem {
    SmemWeights W;
    SmemTile T[kWarps];
    float acc[kAcc];
};

// Forward, loss and gradients of the mean squared error over `count` samples; the gradient
// (kParams fp32, zeroed by the caller) and the summed squared error accumulate in `grad` and
// `loss`. `norm` is the sample count the mean is taken over.
__global__ void __launch_bounds__(kThreads)
k_mlp_gradients(const float *x, const float *target, uint32_t count, float norm,
                const __nv_bfloat16 *wb, const float *master, float *grad, float *loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &G = *reinterpret_cast<GradSmem *>(smem_raw);
    SmemWeights &W = G.W;
    float *acc = G.acc;
    for (int i = threadIdx.x; i < kAcc; i += blockDim.x) {
        acc[i] = 0.0f;
    }
    load_weights(W, wb, master);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t tiles = (count + kTile - 1) / kTile;
    const float scale = 2.0f / norm;
    float sq = 0.0f;
    SmemTile &S = G.T[warp];
    for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles; tile += gridDim.x * kWarps) {
        const uint32_t row0 = tile * kTile;
        Forward F;
        forward(W, x, count, row0, g, t, F);
        // dY = 2 (y - target) / norm on the valid rows and outputs.
        float dy[4];
        const int c = 2 * t;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t r = row0 + g + (i >= 2 ? 8u : 0u);
            const int col = c + (i & 1);
            const bool valid = r < count && col < kOut;
            const float e = valid ? F.y[i] - target[(size_t)r * kOut + col] : 0.0f;
            sq += e * e;
            dy[i] = e * scale;
        }
        // Output layer: dW4 = dY^T h3, db4 = sum dY; dH3 = dY W4.
        __syncwarp();
        for (int i = lane; i < kTile * kHidRow; i += 32) {
            (&S.dz[0][0])[i] = __float2bfloat16(0.0f);
        }
        __syncwarp();
        S.dz[g][c] = __float2bfloat16(dy[0]);
        S.dz[g][c + 1] = __float2bfloat16(dy[1]);
        S.dz[g + 8][c] = __float2bfloat16(dy[2]);
        S.dz[g + 8][c + 1] = __float2bfloat16(dy[3]);
        store_a(S.h, F.a3, g, t);
        __syncwarp();
        weight_grad<kOut, kHid>(S.dz, S.h, acc + kAccW4, g, t);
        if (c < kOut) {
            atomicAdd(&acc[kAccB4 + c], dy[0] + dy[2]);
        }
        if (c + 1 < kOut) {
            atomicAdd(&acc[kAccB4 + c + 1], dy[1] + dy[3]);
        }
        uint32_t dz_out[4];
        dz_out[0] = pack_bf16(dy[0], dy[1]);
        dz_out[1] = pack_bf16(dy[2], dy[3]);
        dz_out[2] = pack_bf16(0.0f, 0.0f);
        dz_out[3] = pack_bf16(0.0f, 0.0f);
        float d[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.0f;
            const uint32_t b0 = pair(&W.w4t[nt * 8 + g][2 * t]);
            const uint32_t b1 = pair(&W.w4t[nt * 8 + g][2 * t + 8]);
            mma(d[nt], dz_out, b0, b1);
        }
        // Layer 3: dZ3 = dH3 * relu'(z3); dW3 = dZ3^T h2; dH2 = dZ3 W3.
        uint32_t dz3[4][4];
        mask_to_a(d, F.m3, dz3);
        __syncwarp();
        store_tile(S.dz, d, g, t);
        store_a(S.h, F.a2, g, t);
        __syncwarp();
        weight_grad<kHid, kHid>(S.dz, S.h, acc + kAccW3, g, t);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            atomicAdd(&acc[kAccB3 + nt * 8 + c], d[nt][0] + d[nt][2]);
            atomicAdd(&acc[kAccB3 + nt * 8 + c + 1], d[nt][1] + d[nt][3]);
        }
        back_mm(dz3, W.w3t, g, t, d);
        // Layer 2.
        uint32_t dz2[4][4];
        mask_to_a(d, F.m2, dz2);
        __syncwarp();
        store_tile(S.dz, d, g, t);
        store_a(S.h, F.a1, g, t);
        __syncwarp();
        weight_grad<kHid, kHid>(S.dz, S.h, acc + kAccW2, g, t);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            atomicAdd(&acc[kAccB2 + nt * 8 + c], d[nt][0] + d[nt][2]);
            atomicAdd(&acc[kAccB2 + nt * 8 + c + 1], d[nt][1] + d[nt][3]);
        }
        back_mm(dz2, W.w2t, g, t, d);
        // Layer 1: dZ1 = dH1 * relu'(z1); dW1 = dZ1^T x.
        uint32_t dz1[4][4];
        mask_to_a(d, F.m1, dz1);
        __syncwarp();
        store_tile(S.dz, d, g, t);
        for (int i = lane; i < kTile * kHidRow; i += 32) {
            (&S.h[0][0])[i] = __float2bfloat16(0.0f);
        }
        __syncwarp();
        *reinterpret_cast<uint32_t *>(&S.h[g][2 * t]) = F.a0[0];
        *reinterpret_cast<uint32_t *>(&S.h[g + 8][2 * t]) = F.a0[1];
        *reinterpret_cast<uint32_t *>(&S.h[g][2 * t + 8]) = F.a0[2];
        *reinterpret_cast<uint32_t *>(&S.h[g + 8][2 * t + 8]) = F.a0[3];
        __syncwarp();
        weight_grad<kHid, kIn>(S.dz, S.h, acc + kAccW1, g, t);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            atomicAdd(&acc[kAccB1 + nt * 8 + c], d[nt][0] + d[nt][2]);
            atomicAdd(&acc[kAccB1 + nt * 8 + c + 1], d[nt][1] + d[nt][3]);
        }
        (void)dz1;
    }
    // The block's sums, once per block.
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, 16);
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, 8);
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, 4);
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, 2);
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, 1);
    if (lane == 0) {
        atomicAdd(loss, sq);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        const float v = acc[acc_index(i)];
        if (v != 0.0f) {
            atomicAdd(&grad[i], v);
        }
    }
}

// Adam on the FP32 master weights (Kingma and Ba, 2015), refreshing the BF16 copies.
__global__ void k_adam(float *master, __nv_bfloat16 *wb, const float *grad, float *m, float *v,
                       float lr, float beta1, float beta2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) {
        return;
    }
    const float gi = grad[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float p = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    master[i] = p;
    wb[i] = __float2bfloat16(p);
}

__global__ void k_refresh_bf16(const float *master, __nv_bfloat16 *wb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) {
        wb[i] = __float2bfloat16(master[i]);
    }
}

} // namespace

struct NphGpuMlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *master = nullptr;     // kParams fp32
    __nv_bfloat16 *wb = nullptr; // kParams bf16
    float *grad = nullptr;
    float *m = nullptr, *v = nullptr;
    float *loss = nullptr;       // 1 float
    float *x = nullptr, *y = nullptr, *tgt = nullptr;
    uint64_t cap = 0;            // samples the staging buffers hold
    uint64_t step = 0;           // Adam's step count
    int sms = 148;
};

namespace {

NphGpuResult mlp_cuda(cudaError_t e)
{
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    return e == cudaErrorMemoryAllocation ? NPH_GPU_OUT_OF_MEMORY : NPH_GPU_DEVICE_LOST;
}

NphGpuResult ensure_samples(NphGpuMlp *n, uint64_t count)
{
    if (count <= n->cap) {
        return NPH_GPU_OK;
    }
    cudaFree(n->x);
    cudaFree(n->y);
    cudaFree(n->tgt);
    n->x = n->y = n->tgt = nullptr;
    n->cap = 0;
    const uint64_t cap = count + count / 4 + 64;
    if (cudaMalloc((void **)&n->x, cap * kIn * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->y, cap * kOut * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&n->tgt, cap * kOut * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    n->cap = cap;
    return NPH_GPU_OK;
}

uint32_t mlp_grid(const NphGpuMlp *n, uint64_t count, uint32_t per_sm)
{
    const uint64_t tiles = (count + kTile - 1) / kTile;
    const uint64_t blocks = (tiles + kWarps - 1) / kWarps;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)n->sms * per_sm));
}

// Zeroes the gradient and loss accumulators and accumulates those of `count` samples at x/t.
void enqueue_gradients(NphGpuMlp *n, const float *x, const float *t, uint32_t count, float norm)
{
    cudaMemsetAsync(n->grad, 0, kParams * sizeof(float), n->stream);
    cudaMemsetAsync(n->loss, 0, sizeof(float), n->stream);
    k_mlp_gradients<<<mlp_grid(n, count, 2), kThreads, sizeof(GradSmem), n->stream>>>(x, t, count, norm, n->wb,
                                                                                      n->master, n->grad, n->loss);
}

// Uniform(-a, a) initial weights (a = sqrt(6 / fan_in)), the output layer scaled by 0.1, zero
// biases, from a splitmix64 stream.
void init_weights(std::vector<float> &w, uint64_t seed)
{
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    w.assign(kParams, 0.0f);
    auto fill = [&](int off, int fan_out, int fan_in, double scale) {
        const double a = scale * std::sqrt(6.0 / fan_in);
        for (int i = 0; i < fan_out * fan_in; ++i) {
            w[off + i] = (float)((2.0 * next() - 1.0) * a);
        }
    };
    fill(kW1, kHid, kIn, 1.0);
    fill(kW2, kHid, kHid, 1.0);
    fill(kW3, kHid, kHid, 1.0);
    fill(kW4, kOut, kHid, 0.1);
}

} // namespace

// A seeded pattern in [-1, 1): a splitmix64 hash of (seed, i).
__global__ void k_fill_pattern(float *p, uint64_t n, uint64_t seed)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = (seed + i + 1u) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        p[i] = (float)(z >> 40) * (2.0f / 16777216.0f) - 1.0f;
    }
}

// The network's inference on device features (the solver's learned warm start).
void nph_mlp_forward_device(const NphGpuMlp *n, const float *x, uint32_t count, float *y, cudaStream_t st)
{
    if (count == 0) {
        return;
    }
    k_mlp_forward<<<mlp_grid(n, count, 8), kThreads, 0, st>>>(x, count, nullptr, n->wb, n->master, y);
}

void nph_mlp_forward_device_count(const NphGpuMlp *n, const float *x, const uint32_t *count_dev,
                                  uint32_t max_count, float *y, cudaStream_t st)
{
    if (max_count == 0) {
        return;
    }
    k_mlp_forward<<<mlp_grid(n, max_count, 8), kThreads, 0, st>>>(x, max_count, count_dev, n->wb, n->master, y);
}

int nph_mlp_device(const NphGpuMlp *n) { return n->device; }

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_mlp_create(int32_t device, uint64_t seed, NphGpuMlp **out)
{
    if (out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    if (device < 0 || device >= count) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(device);
    if (cudaFuncSetAttribute(k_mlp_gradients, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(GradSmem)) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    NphGpuMlp *n = new (std::nothrow) NphGpuMlp();
    if (n == nullptr) {
        return NPH_GPU_OUT_OF_MEMORY;
    }
    n->device = device;
    cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, device);
    const bool ok = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaMalloc((void **)&n->master, kParams * sizeof(float)) == cudaSuccess &&
                    cudaMalloc((void **)&n->wb, kParams * sizeof(__nv_bfloat16)) == cudaSuccess &&
                    cudaMalloc((void **)&n->grad, kParams * sizeof(float)) == cudaSuccess &&
                    cudaMalloc((void **)&n->m, kParams * sizeof(float)) == cudaSuccess &&
                    cudaMalloc((void **)&n->v, kParams * sizeof(float)) == cudaSuccess &&
                    cudaMalloc((void **)&n->loss, sizeof(float)) == cudaSuccess;
    if (!ok) {
        nph_gpu_mlp_destroy(n);
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    std::vector<float> w;
    init_weights(w, seed);
    const NphGpuResult r = nph_gpu_mlp_set_weights(n, w.data());
    if (r != NPH_GPU_OK) {
        nph_gpu_mlp_destroy(n);
        return r;
    }
    *out = n;
    return NPH_GPU_OK;
}

NPH_GPU_API void nph_gpu_mlp_destroy(NphGpuMlp *n)
{
    if (n == nullptr) {
        return;
    }
    cudaSetDevice(n->device);
    if (n->stream != nullptr) {
        cudaStreamSynchronize(n->stream);
        cudaStreamDestroy(n->stream);
    }
    cudaFree(n->master);
    cudaFree(n->wb);
    cudaFree(n->grad);
    cudaFree(n->m);
    cudaFree(n->v);
    cudaFree(n->loss);
    cudaFree(n->x);
    cudaFree(n->y);
    cudaFree(n->tgt);
    delete n;
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_set_weights(NphGpuMlp *n, const float *params)
{
    if (n == nullptr || params == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    cudaMemcpyAsync(n->master, params, kParams * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    cudaMemsetAsync(n->m, 0, kParams * sizeof(float), n->stream);
    cudaMemsetAsync(n->v, 0, kParams * sizeof(float), n->stream);
    k_refresh_bf16<<<(kParams + 255) / 256, 256, 0, n->stream>>>(n->master, n->wb);
    n->step = 0;
    return mlp_cuda(cudaStreamSynchronize(n->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_get_weights(const NphGpuMlp *n, float *params)
{
    if (n == nullptr || params == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    cudaMemcpyAsync(params, n->master, kParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    return mlp_cuda(cudaStreamSynchronize(n->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_predict(NphGpuMlp *n, const float *features, uint64_t count,
                                             float *out)
{
    if (n == nullptr || (count > 0 && (features == nullptr || out == nullptr)) || count > 0xFFFFFFFFull) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    NphGpuResult r = ensure_samples(n, count);
    if (r != NPH_GPU_OK || count == 0) {
        return r;
    }
    cudaMemcpyAsync(n->x, features, count * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    nph_mlp_forward_device(n, n->x, (uint32_t)count, n->y, n->stream);
    cudaMemcpyAsync(out, n->y, count * kOut * sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    return mlp_cuda(cudaStreamSynchronize(n->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_gradients(NphGpuMlp *n, const float *features,
                                               const float *targets, uint64_t count, float *grad,
                                               float *loss)
{
    if (n == nullptr || count == 0 || features == nullptr || targets == nullptr || grad == nullptr ||
        count > 0xFFFFFFFFull) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    NphGpuResult r = ensure_samples(n, count);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaMemcpyAsync(n->x, features, count * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    cudaMemcpyAsync(n->tgt, targets, count * kOut * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    enqueue_gradients(n, n->x, n->tgt, (uint32_t)count, (float)count);
    cudaMemcpyAsync(grad, n->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    float sq = 0.0f;
    cudaMemcpyAsync(&sq, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    r = mlp_cuda(cudaStreamSynchronize(n->stream));
    if (loss != nullptr) {
        *loss = sq / (float)count;
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_time_kernels(NphGpuMlp *n, uint64_t count, uint32_t reps, float *forward_ms,
                                                  float *gradients_ms)
{
    if (n == nullptr || count == 0 || count > 0x80000000ull || reps == 0 || forward_ms == nullptr ||
        gradients_ms == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    NphGpuResult r = ensure_samples(n, count);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const uint32_t fill_blocks = (uint32_t)n->sms * 8u;
    k_fill_pattern<<<fill_blocks, 256, 0, n->stream>>>(n->x, count * kIn, 1u);
    k_fill_pattern<<<fill_blocks, 256, 0, n->stream>>>(n->tgt, count * kOut, 2u);
    cudaEvent_t e[3];
    for (cudaEvent_t &ev : e) {
        cudaEventCreate(&ev);
    }
    const uint32_t c = (uint32_t)count;
    nph_mlp_forward_device(n, n->x, c, n->y, n->stream); // warm-up launches
    enqueue_gradients(n, n->x, n->tgt, c, (float)count);
    cudaEventRecord(e[0], n->stream);
    for (uint32_t i = 0; i < reps; ++i) {
        nph_mlp_forward_device(n, n->x, c, n->y, n->stream);
    }
    cudaEventRecord(e[1], n->stream);
    for (uint32_t i = 0; i < reps; ++i) {
        enqueue_gradients(n, n->x, n->tgt, c, (float)count);
    }
    cudaEventRecord(e[2], n->stream);
    r = mlp_cuda(cudaStreamSynchronize(n->stream));
    float f = 0.0f, g = 0.0f;
    if (r == NPH_GPU_OK) {
        cudaEventElapsedTime(&f, e[0], e[1]);
        cudaEventElapsedTime(&g, e[1], e[2]);
    }
    for (cudaEvent_t &ev : e) {
        cudaEventDestroy(ev);
    }
    *forward_ms = f / (float)reps;
    *gradients_ms = g / (float)reps;
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_mlp_train(NphGpuMlp *n, const float *features, const float *targets,
                                           uint64_t count, uint32_t epochs, uint32_t batch, float lr,
                                           uint64_t shuffle_seed, float *final_loss)
{
    if (n == nullptr || count == 0 || features == nullptr || targets == nullptr || batch == 0 ||
        count > 0xFFFFFFFFull || !(lr > 0.0f)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(n->device);
    NphGpuResult r = ensure_samples(n, count);
    if (r != NPH_GPU_OK) {
        return r;
    }
    // The samples in a seeded shuffled order (Fisher-Yates over xorshift64), once on the
    // device; each epoch walks that order's mini-batches from a seeded starting batch.
    std::vector<uint32_t> perm(count);
    for (uint64_t i = 0; i < count; ++i) {
        perm[i] = (uint32_t)i;
    }
    uint64_t s = shuffle_seed * 0x9E3779B97F4A7C15ull + 7;
    auto rnd = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    };
    for (uint64_t i = count - 1; i > 0; --i) {
        std::swap(perm[i], perm[rnd() % (i + 1)]);
    }
    std::vector<float> xs(count * kIn), ts(count * kOut);
    for (uint64_t i = 0; i < count; ++i) {
        std::memcpy(&xs[i * kIn], &features[(size_t)perm[i] * kIn], kIn * sizeof(float));
        std::memcpy(&ts[i * kOut], &targets[(size_t)perm[i] * kOut], kOut * sizeof(float));
    }
    cudaMemcpyAsync(n->x, xs.data(), count * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    cudaMemcpyAsync(n->tgt, ts.data(), count * kOut * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    const uint64_t batches = (count + batch - 1) / batch;
    for (uint32_t e = 0; e < epochs; ++e) {
        const uint64_t shift = rnd() % batches;
        for (uint64_t bi = 0; bi < batches; ++bi) {
            const uint64_t b = (bi + shift) % batches;
            const uint64_t first = b * batch;
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(batch, count - first);
            enqueue_gradients(n, n->x + first * kIn, n->tgt + first * kOut, cnt, (float)cnt);
            n->step += 1;
            const float c1 = 1.0f - std::pow(beta1, (float)n->step);
            const float c2 = 1.0f - std::pow(beta2, (float)n->step);
            k_adam<<<(kParams + 255) / 256, 256, 0, n->stream>>>(n->master, n->wb, n->grad, n->m, n->v, lr,
                                                                 beta1, beta2, eps, c1, c2);
        }
    }
    // The loss over all samples with the final weights.
    enqueue_gradients(n, n->x, n->tgt, (uint32_t)count, (float)count);
    float sq = 0.0f;
    cudaMemcpyAsync(&sq, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    r = mlp_cuda(cudaStreamSynchronize(n->stream));
    if (r == NPH_GPU_OK && final_loss != nullptr) {
        *final_loss = sq / (float)count;
    }
    return r;
}

} // extern "C"
