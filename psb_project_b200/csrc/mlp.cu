// mlp.cu -- learned pressure warm start for the PCISPH corrector.
//
// A per-particle MLP predicts each step's initial pressure so that the
// eta-controlled corrector (unchanged; it still iterates to the same eta and
// decides convergence) starts closer to the converged pressure. The
// reference has no counterpart: it starts every step from p = 0
// (PciSphSystem_Kernel.cu:131).
//
// Two networks, chosen per context (psb_mlp_set_arch):
//   PSB_MLP_SILU6  6 -> 64 -> 64 -> 1, SiLU: the configured network, inputs f0..f5;
//   PSB_MLP_RELU7  7 -> 64 -> 64 -> 1, ReLU: adds f6.
// Inputs, computed at the step's start positions from the neighbour list
// (by the density pass at x, k_density_x in sph.cu):
//   f0 neighbour count / 32
//   f1 advected density (rho - dt rho div v - rho0)/rho0 * 100
//   f2 velocity divergence div v * dt * 100, div v = sum (m/rho0)(v_j - v_i).gradW_ij
//   f3 previous-step pressure / p_scale
//   f4 distance to the nearest box face / h, capped at 1
//   f5 |sum m gradW_ij| * h / rho0 (density-gradient magnitude)
//   f6 previous-step pressure smoothed with the poly6 weights / p_scale
// Output y: initial pressure max(0, y) * p_scale, p_scale = rho0 |g| 0.1 m.
//
// Precision: weights and activations are BF16 (round-to-nearest-even at
// every stored activation), accumulation FP32, master weights FP32 (Adam).
// SiLU is z sigma(z) = z/2 (1 + tanh(z/2)) with the hardware tanh
// approximation (tanh.approx.f32, one special-function op per unit); its
// error is below the BF16 rounding the activation then takes.
//
// Training is on the GPU, on tensor cores: (features, converged pressure)
// pairs are collected from steps of the same eta-loop, then minibatch Adam
// on an MSE loss. One fused kernel runs forward and backward over tiles of
// 64 samples per block with mma.sync (BF16 in, FP32 accumulate): the two
// forward layers, the back-propagation through W2, and the weight
// gradients of W1 and W2 as products over the tile's samples. Bias and
// output-layer gradients are FP32 sums reduced with warp shuffles.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "psb.h"
#include "psb_internal.cuh"

namespace psb {

namespace {

constexpr int kH = 64;

// Parameter layout: W1[64][NIN], b1[64], W2[64][64], b2[64], w3[64], b3.
template <int NIN>
struct Layout {
    static constexpr int W1 = 0, B1 = W1 + kH * NIN, W2 = B1 + kH, B2 = W2 + kH * kH, W3 = B2 + kH, B3 = W3 + kH,
                         N = B3 + 1;
};
static_assert(Layout<7>::N == kMlpParams, "the largest network's parameter count");
static_assert(Layout<6>::N == 4673, "the configured network's parameter count");

enum { kSilu = 0, kRelu = 1 };

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

template <int ACT>
__device__ __forceinline__ float act(float z) {
    if (ACT == kRelu) return fmaxf(z, 0.f);
    const float hz = 0.5f * z;
    return fmaf(hz, tanh_approx(hz), hz);         // z sigma(z) = z/2 (1 + tanh(z/2))
}

template <int ACT>
__device__ __forceinline__ float act_grad(float z) {
    if (ACT == kRelu) return z > 0.f ? 1.f : 0.f;
    const float s = fmaf(0.5f, tanh_approx(0.5f * z), 0.5f);    // sigma(z)
    return s * fmaf(z, 1.f - s, 1.f);                            // sigma (1 + z (1 - sigma))
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A B + D, m16n8k16, A row-major 16 x 16 and B column-major 16 x 8 in
// BF16, D in FP32. Fragments (lane = 4 gid + tig): a0 (gid, 2tig..+1),
// a1 (gid+8, 2tig..+1), a2 (gid, 2tig+8..+9), a3 (gid+8, 2tig+8..+9);
// b0 (k 2tig..+1, n gid), b1 (k 2tig+8..+9, n gid); d0..d3 (gid, 2tig),
// (gid, 2tig+1), (gid+8, 2tig), (gid+8, 2tig+1).
__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-memory weight images. W1 rows hold 8 BF16 (NIN used, zero padded),
// as B fragments of layer 1 (n = unit, k = input). W2 rows are padded to 36
// words so that the eight groups of a fragment load fall in distinct banks.
constexpr int kW1Stride = 4;      // 32-bit words per W1 row
constexpr int kRow = 36;          // 32-bit words per padded row of 64 BF16

template <int NIN>
__device__ __forceinline__ void stage_weights(const __nv_bfloat16* __restrict__ w, uint32_t* sW1, uint32_t* sW2,
                                              uint32_t* sW2T, float* sB1, float* sB2, float* sW3, float* sB3) {
    using L = Layout<NIN>;
    for (int i = threadIdx.x; i < kH * kW1Stride; i += blockDim.x) {
        const int r = i / kW1Stride, k = 2 * (i % kW1Stride);
        const float lo = k < NIN ? __bfloat162float(w[L::W1 + r * NIN + k]) : 0.f;
        const float hi = k + 1 < NIN ? __bfloat162float(w[L::W1 + r * NIN + k + 1]) : 0.f;
        sW1[i] = pack_bf16(lo, hi);
    }
    for (int i = threadIdx.x; i < kH * 32; i += blockDim.x) {
        const int r = i / 32, k = 2 * (i % 32);
        sW2[r * kRow + i % 32] = pack_bf16(__bfloat162float(w[L::W2 + r * kH + k]), __bfloat162float(w[L::W2 + r * kH + k + 1]));
        if (sW2T)       // [k][j]: pairs along j (rows of W2)
            sW2T[r * kRow + i % 32] =
                pack_bf16(__bfloat162float(w[L::W2 + k * kH + r]), __bfloat162float(w[L::W2 + (k + 1) * kH + r]));
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        sB1[i] = __bfloat162float(w[L::B1 + i]);
        sB2[i] = __bfloat162float(w[L::B2 + i]);
        sW3[i] = __bfloat162float(w[L::W3 + i]);
    }
    if (threadIdx.x == 0) *sB3 = __bfloat162float(w[L::B3]);
}

// Layer 1 of a 16-row tile: z1 = x W1^T + b1 (accumulator layout).
__device__ __forceinline__ void layer1(float (&z1)[8][4], uint32_t a0, uint32_t a1, const uint32_t* sW1,
                                       const float* sB1, int gid, int tig) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + 2 * tig;
        z1[nt][0] = sB1[col]; z1[nt][1] = sB1[col + 1];
        z1[nt][2] = sB1[col]; z1[nt][3] = sB1[col + 1];
        mma_bf16(z1[nt], a0, a1, 0u, 0u, sW1[(nt * 8 + gid) * kW1Stride + tig], 0u);
    }
}

// The accumulator fragments of a 16 x 64 product, through f and rounded to
// BF16, are the A fragments of the next 16 x 64 x K product (K-step ks:
// n-tiles 2 ks and 2 ks + 1).
template <class F>
__device__ __forceinline__ void to_a_frags(uint32_t (&a)[4][4], const float (&z)[8][4], F&& f) {
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        a[ks][0] = pack_bf16(f(z[2 * ks][0]), f(z[2 * ks][1]));
        a[ks][1] = pack_bf16(f(z[2 * ks][2]), f(z[2 * ks][3]));
        a[ks][2] = pack_bf16(f(z[2 * ks + 1][0]), f(z[2 * ks + 1][1]));
        a[ks][3] = pack_bf16(f(z[2 * ks + 1][2]), f(z[2 * ks + 1][3]));
    }
}

// 16 x 64 = A (16 x 64, fragments) B, B(k, n) the 32-bit pairs along k of
// rows n of a padded image (W2 for the forward, W2^T for the backward).
__device__ __forceinline__ void layer64(float (&z)[8][4], const uint32_t (&a)[4][4], const uint32_t* sB,
                                        const float* bias, int gid, int tig) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + 2 * tig;
        if (bias) {
            z[nt][0] = bias[col]; z[nt][1] = bias[col + 1];
            z[nt][2] = bias[col]; z[nt][3] = bias[col + 1];
        } else {
            z[nt][0] = z[nt][1] = z[nt][2] = z[nt][3] = 0.f;
        }
        const uint32_t* row = sB + (nt * 8 + gid) * kRow;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
            mma_bf16(z[nt], a[ks][0], a[ks][1], a[ks][2], a[ks][3], row[8 * ks + tig], row[8 * ks + 4 + tig]);
    }
}

// ---- inference -----------------------------------------------------------------
// One warp evaluates 16 particles per pass: layer 1 a [16 x 16] x [16 x 64]
// product (the inputs zero padded), layer 2 [16 x 64] x [64 x 64] from
// layer 1's accumulators, the output layer a per-thread dot product finished
// with two shuffles.
// y_raw != nullptr: write the raw output y there (host-facing evaluation)
// instead of the initial pressure max(0, y) p_scale into rp.
template <int NIN, int ACT>
__global__ void __launch_bounds__(256) k_mlp_infer_mma(int n, const float* __restrict__ feats,
                                                       const __nv_bfloat16* __restrict__ w, float p_scale,
                                                       float2* __restrict__ rp, float* __restrict__ y_raw) {
    __shared__ uint32_t sW1[kH * kW1Stride];
    __shared__ uint32_t sW2[kH * kRow];
    __shared__ float sB1[kH], sB2[kH], sW3[kH];
    __shared__ float sB3;
    stage_weights<NIN>(w, sW1, sW2, nullptr, sB1, sB2, sW3, &sB3);
    __syncthreads();

    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    for (int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n; tile += warps_total) {
        const int r0 = tile * 16 + gid, r1 = r0 + 8;
        uint32_t a0 = 0u, a1 = 0u;
        {
            const int k = 2 * tig;
            if (k < NIN) {
                const float f00 = r0 < n ? feats[(size_t)r0 * 8 + k] : 0.f;
                const float f01 = r0 < n && k + 1 < NIN ? feats[(size_t)r0 * 8 + k + 1] : 0.f;
                const float f10 = r1 < n ? feats[(size_t)r1 * 8 + k] : 0.f;
                const float f11 = r1 < n && k + 1 < NIN ? feats[(size_t)r1 * 8 + k + 1] : 0.f;
                a0 = pack_bf16(f00, f01);
                a1 = pack_bf16(f10, f11);
            }
        }
        float z[8][4];
        layer1(z, a0, a1, sW1, sB1, gid, tig);
        uint32_t h1[4][4];
        to_a_frags(h1, z, [](float v) { return act<ACT>(v); });
        layer64(z, h1, sW2, sB2, gid, tig);
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {     // output layer on the BF16-rounded activations
            const int col = nt * 8 + 2 * tig;
            const float w30 = sW3[col], w31 = sW3[col + 1];
            y0 = fmaf(w30, bf(act<ACT>(z[nt][0])), y0);
            y0 = fmaf(w31, bf(act<ACT>(z[nt][1])), y0);
            y1 = fmaf(w30, bf(act<ACT>(z[nt][2])), y1);
            y1 = fmaf(w31, bf(act<ACT>(z[nt][3])), y1);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (tig == 0) {
            if (y_raw) {
                if (r0 < n) y_raw[r0] = y0 + sB3;
                if (r1 < n) y_raw[r1] = y1 + sB3;
            } else {
                if (r0 < n) rp[r0].y = fmaxf(0.f, y0 + sB3) * p_scale;
                if (r1 < n) rp[r1].y = fmaxf(0.f, y1 + sB3) * p_scale;
            }
        }
    }
}

// ---- training ---------------------------------------------------------------------
constexpr int kTrainWarps = 4;
constexpr int kTrainRows = 16 * kTrainWarps;    // samples per block tile
constexpr int kTRow = 72;                       // BF16 per padded row of a transposed activation tile
constexpr int kPartStride = kMlpParams + 1;     // floats per block row of the gradient partials

// Shared memory of the training kernel (dynamic): weight images, and per
// tile the BF16 activations transposed (row = unit, column = sample), the
// operands of the weight-gradient products.
struct TrainSmem {
    uint32_t W1[kH * kW1Stride];
    uint32_t W2[kH * kRow];
    uint32_t W2T[kH * kRow];
    float B1[kH], B2[kH], W3[kH], B3;
    float G[kTrainWarps][3 * kH + 2];           // per warp: gradients of b1, b2, w3; b3; the loss
    __nv_bfloat16 H1T[kH * kTRow];              // h1[k][m]
    __nv_bfloat16 D2T[kH * kTRow];              // dz2[j][m]
    __nv_bfloat16 D1T[kH * kTRow];              // dz1[k][m]
    __nv_bfloat16 XT[8 * kTRow];                // x[i][m]
};

__device__ __forceinline__ uint32_t word(const __nv_bfloat16* base, int row, int col) {
    return *reinterpret_cast<const uint32_t*>(base + row * kTRow + col);
}

// Column sums of a 16 x 64 accumulator tile over its 16 rows: every lane
// ends with the sums of its columns (nt, 2 tig + c).
__device__ __forceinline__ float row_sum(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// Mean-squared-error loss and its gradient over `batch` samples (sample b:
// row sel[b] of X (stride 8) and T, or row b without sel). Each block
// writes its partial sums -- every parameter's gradient at its layout
// index, the loss at kMlpParams -- to its own row of `partial` (kPartStride
// floats); k_grad_reduce adds the rows in block order. No atomics: the
// gradient, and so the trained network, is the same bits on every run.
template <int NIN, int ACT>
__global__ void __launch_bounds__(kTrainWarps * 32) k_mlp_train_mma(int batch, const float* __restrict__ X,
                                                                  const float* __restrict__ T,
                                                                  const uint32_t* __restrict__ sel,
                                                                  const __nv_bfloat16* __restrict__ w,
                                                                  float* __restrict__ partial) {
    using L = Layout<NIN>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    stage_weights<NIN>(w, S.W1, S.W2, S.W2T, S.B1, S.B2, S.W3, &S.B3);
    for (int i = threadIdx.x; i < kTrainWarps * (3 * kH + 2); i += blockDim.x) (&S.G[0][0])[i] = 0.f;
    __syncthreads();

    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3, wp = threadIdx.x >> 5;
    const float inv_b = 1.f / (float)batch;
    float gW2[8][4], gW1[4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) gW2[nt][0] = gW2[nt][1] = gW2[nt][2] = gW2[nt][3] = 0.f;
    gW1[0] = gW1[1] = gW1[2] = gW1[3] = 0.f;
    float g_b3 = 0.f, g_loss = 0.f;

    for (int tile = blockIdx.x; tile * kTrainRows < batch; tile += gridDim.x) {
        const int m0 = wp * 16 + gid, m1 = m0 + 8;                 // rows of this warp in the block tile
        const int r0 = tile * kTrainRows + m0, r1 = r0 + 8;
        const bool v0 = r0 < batch, v1 = r1 < batch;
        const uint32_t row0 = v0 ? (sel ? sel[r0] : (uint32_t)r0) : 0u;
        const uint32_t row1 = v1 ? (sel ? sel[r1] : (uint32_t)r1) : 0u;
        const int k = 2 * tig;
        const float x00 = v0 && k < NIN ? bf(X[(size_t)row0 * 8 + k]) : 0.f;
        const float x01 = v0 && k + 1 < NIN ? bf(X[(size_t)row0 * 8 + k + 1]) : 0.f;
        const float x10 = v1 && k < NIN ? bf(X[(size_t)row1 * 8 + k]) : 0.f;
        const float x11 = v1 && k + 1 < NIN ? bf(X[(size_t)row1 * 8 + k + 1]) : 0.f;
        // ---- forward
        float z1[8][4];
        layer1(z1, pack_bf16(x00, x01), pack_bf16(x10, x11), S.W1, S.B1, gid, tig);
        uint32_t a[4][4];
        to_a_frags(a, z1, [](float v) { return act<ACT>(v); });
        float z2[8][4];
        layer64(z2, a, S.W2, S.B2, gid, tig);
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int col = nt * 8 + 2 * tig;
            y0 = fmaf(S.W3[col], bf(act<ACT>(z2[nt][0])), y0);
            y0 = fmaf(S.W3[col + 1], bf(act<ACT>(z2[nt][1])), y0);
            y1 = fmaf(S.W3[col], bf(act<ACT>(z2[nt][2])), y1);
            y1 = fmaf(S.W3[col + 1], bf(act<ACT>(z2[nt][3])), y1);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        const float e0 = v0 ? y0 + S.B3 - T[row0] : 0.f;
        const float e1 = v1 ? y1 + S.B3 - T[row1] : 0.f;
        const float dy0 = 2.f * e0 * inv_b, dy1 = 2.f * e1 * inv_b;   // d(mean e^2)/dy
        if (tig == 0) {
            g_b3 += dy0 + dy1;
            g_loss += (e0 * e0 + e1 * e1) * inv_b;
        }
        // ---- output layer and second hidden layer: dz2 = dy w3 act'(z2)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int col = nt * 8 + 2 * tig + c;
                const float gw3 = row_sum(dy0 * bf(act<ACT>(z2[nt][c])) + dy1 * bf(act<ACT>(z2[nt][2 + c])));
                const float d0 = dy0 * S.W3[col] * act_grad<ACT>(z2[nt][c]);
                const float d1 = dy1 * S.W3[col] * act_grad<ACT>(z2[nt][2 + c]);
                const float gb2 = row_sum(d0 + d1);
                if (gid == 0) {         // one lane per column in the warp
                    S.G[wp][2 * kH + col] += gw3;
                    S.G[wp][kH + col] += gb2;
                }
                z2[nt][c] = d0;
                z2[nt][2 + c] = d1;
            }
        }
        // ---- first hidden layer: dz1 = (dz2 W2) act'(z1)
        to_a_frags(a, z2, [](float v) { return v; });
        float dh[8][4];
        layer64(dh, a, S.W2T, nullptr, gid, tig);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int col = nt * 8 + 2 * tig + c;
                const float d0 = dh[nt][c] * act_grad<ACT>(z1[nt][c]);
                const float d1 = dh[nt][2 + c] * act_grad<ACT>(z1[nt][2 + c]);
                const float gb1 = row_sum(d0 + d1);
                if (gid == 0) S.G[wp][col] += gb1;
                // the tile's operands of the weight-gradient products, transposed
                S.H1T[col * kTRow + m0] = __float2bfloat16_rn(act<ACT>(z1[nt][c]));
                S.H1T[col * kTRow + m1] = __float2bfloat16_rn(act<ACT>(z1[nt][2 + c]));
                S.D2T[col * kTRow + m0] = __float2bfloat16_rn(z2[nt][c]);
                S.D2T[col * kTRow + m1] = __float2bfloat16_rn(z2[nt][2 + c]);
                S.D1T[col * kTRow + m0] = __float2bfloat16_rn(d0);
                S.D1T[col * kTRow + m1] = __float2bfloat16_rn(d1);
            }
        }
        S.XT[k * kTRow + m0] = __float2bfloat16_rn(x00);
        S.XT[(k + 1) * kTRow + m0] = __float2bfloat16_rn(x01);
        S.XT[k * kTRow + m1] = __float2bfloat16_rn(x10);
        S.XT[(k + 1) * kTRow + m1] = __float2bfloat16_rn(x11);
        __syncthreads();
        // ---- weight gradients over the tile's 64 samples: warp wp takes
        // rows [16 wp, 16 wp + 16) of dW2 (= dz2^T h1) and dW1 (= dz1^T x)
        const int j0 = wp * 16;
#pragma unroll
        for (int ks = 0; ks < kTrainRows / 16; ++ks) {
            const int c0 = ks * 16 + 2 * tig;
            const uint32_t a0 = word(S.D2T, j0 + gid, c0), a1 = word(S.D2T, j0 + gid + 8, c0);
            const uint32_t a2 = word(S.D2T, j0 + gid, c0 + 8), a3 = word(S.D2T, j0 + gid + 8, c0 + 8);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
                mma_bf16(gW2[nt], a0, a1, a2, a3, word(S.H1T, nt * 8 + gid, c0), word(S.H1T, nt * 8 + gid, c0 + 8));
            mma_bf16(gW1, word(S.D1T, j0 + gid, c0), word(S.D1T, j0 + gid + 8, c0), word(S.D1T, j0 + gid, c0 + 8),
                     word(S.D1T, j0 + gid + 8, c0 + 8), word(S.XT, gid, c0), word(S.XT, gid, c0 + 8));
        }
        __syncthreads();
    }
    // ---- the block's partial sums: the weight tiles straight from the
    // accumulators (each parameter held by one lane), the rest summed over
    // the warps in order
    float* part = partial + (size_t)blockIdx.x * kPartStride;
    const int j0 = wp * 16;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + 2 * tig;
        part[L::W2 + (j0 + gid) * kH + col] = gW2[nt][0];
        part[L::W2 + (j0 + gid) * kH + col + 1] = gW2[nt][1];
        part[L::W2 + (j0 + gid + 8) * kH + col] = gW2[nt][2];
        part[L::W2 + (j0 + gid + 8) * kH + col + 1] = gW2[nt][3];
    }
    {
        const int i = 2 * tig;
        if (i < NIN) {
            part[L::W1 + (j0 + gid) * NIN + i] = gW1[0];
            part[L::W1 + (j0 + gid + 8) * NIN + i] = gW1[2];
        }
        if (i + 1 < NIN) {
            part[L::W1 + (j0 + gid) * NIN + i + 1] = gW1[1];
            part[L::W1 + (j0 + gid + 8) * NIN + i + 1] = gW1[3];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        g_b3 += __shfl_xor_sync(0xffffffffu, g_b3, o);
        g_loss += __shfl_xor_sync(0xffffffffu, g_loss, o);
    }
    if (lane == 0) {
        S.G[wp][3 * kH] = g_b3;
        S.G[wp][3 * kH + 1] = g_loss;
    }
    __syncthreads();
    auto warp_sum = [&](int i) {
        float v = S.G[0][i];
#pragma unroll
        for (int q = 1; q < kTrainWarps; ++q) v += S.G[q][i];
        return v;
    };
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        part[L::B1 + i] = warp_sum(i);
        part[L::B2 + i] = warp_sum(kH + i);
        part[L::W3 + i] = warp_sum(2 * kH + i);
    }
    if (threadIdx.x == 0) {
        part[L::B3] = warp_sum(3 * kH);
        part[kMlpParams] = warp_sum(3 * kH + 1);
    }
}

// grad[p] (p < np) and the loss: the blocks' partial rows added in a fixed
// order. Warp w of a block adds rows w, w + 8, ... for 32 consecutive
// entries; the eight warp sums are then added in warp order.
__global__ void __launch_bounds__(256) k_grad_reduce(int nblocks, int np, const float* __restrict__ partial,
                                                     float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float s[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int q = blockIdx.x * 32 + lane;                 // q == np: the loss
    const int src = q < np ? q : kMlpParams;
    float v = 0.f;
    if (q <= np) {
#pragma unroll 4
        for (int b = w; b < nblocks; b += 8) v += partial[(size_t)b * kPartStride + src];
    }
    s[w][lane] = v;
    __syncthreads();
    if (w == 0 && q <= np) {
        float t = s[0][lane];
#pragma unroll
        for (int k = 1; k < 8; ++k) t += s[k][lane];
        if (q < np) grad[q] = t;
        else *loss = t;
    }
}

__global__ void k_adam(int np, float* __restrict__ wmaster, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, __nv_bfloat16* __restrict__ wbf, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float g = grad[i];
    const float m = b1 * m1[i] + (1.f - b1) * g;
    const float v = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = m;
    m2[i] = v;
    const float w = wmaster[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    wmaster[i] = w;
    wbf[i] = __float2bfloat16_rn(w);
}

__global__ void k_to_bf16(int np, const float* __restrict__ w, __nv_bfloat16* __restrict__ wbf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) wbf[i] = __float2bfloat16_rn(w[i]);
}

// Samples: uniform over [0, size) from SplitMix64 of (seed, iteration, b).
__global__ void k_sample(int batch, uint64_t size, uint64_t seed, uint32_t* __restrict__ sel) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(b + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    sel[b] = (uint32_t)(z % size);
}

// Appends (features, converged pressure) of every stride-th slot, from
// `offset`, to the dataset rows [base, base + ceil((n - offset)/stride)).
__global__ void k_collect(int n, int stride, int offset, uint64_t base, uint64_t cap, const float* __restrict__ feats,
                          const float2* __restrict__ rp, float p_scale, float* __restrict__ X, float* __restrict__ T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = offset + i * stride;
    if (s >= n) return;
    const uint64_t row = (base + (uint64_t)i) % cap;
    const float* f = feats + (size_t)s * 8;
#pragma unroll
    for (int k = 0; k < 8; ++k) X[row * 8 + k] = f[k];
    T[row] = rp[s].y / p_scale;
}

__global__ void k_zero_pressure(int n, float2* __restrict__ rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rp[i].y = 0.f;
}

inline int grid_of(int n, int b = kBlock) { return (n + b - 1) / b; }

// f(integral_constant NIN, integral_constant ACT) for the network `arch`.
template <class F>
void with_arch(int arch, F&& f) {
    if (arch == PSB_MLP_RELU7) f(std::integral_constant<int, 7>{}, std::integral_constant<int, kRelu>{});
    else f(std::integral_constant<int, 6>{}, std::integral_constant<int, kSilu>{});
}

void infer(cudaStream_t st, int arch, int n, const float* feats, const void* wbf, float p_scale, float2* rp, float* y) {
    if (n <= 0) return;
    const int tiles = (n + 15) / 16;
    const int blocks = std::min((tiles + 7) / 8, 148 * 8);      // 8 warps per block, grid-stride over tiles
    with_arch(arch, [&](auto nin, auto a) {
        k_mlp_infer_mma<decltype(nin)::value, decltype(a)::value>
            <<<blocks, 256, 0, st>>>(n, feats, (const __nv_bfloat16*)wbf, p_scale, rp, y);
    });
}

}  // namespace

int mlp_inputs(int arch) { return arch == PSB_MLP_RELU7 ? 7 : 6; }
int mlp_params(int arch) { return arch == PSB_MLP_RELU7 ? Layout<7>::N : Layout<6>::N; }

void launch_zero_pressure(cudaStream_t st, int n, float2* rp) {
    if (n > 0) k_zero_pressure<<<grid_of(n), kBlock, 0, st>>>(n, rp);
}

void launch_mlp_infer(cudaStream_t st, int arch, int n, const float* feats, const void* wbf, float p_scale,
                      float2* rp) {
    infer(st, arch, n, feats, wbf, p_scale, rp, nullptr);
}

// Host-facing forward through the tensor-core kernel the warm start uses
// (rows of stride 8).
void launch_mlp_forward(cudaStream_t st, int arch, int n, const float* X, const void* wbf, float* y) {
    infer(st, arch, n, X, wbf, 1.f, nullptr, y);
}

void launch_mlp_grad(cudaStream_t st, int arch, int batch, const float* X, const float* T, const uint32_t* sel,
                     const void* wbf, float* partial, float* grad, float* loss) {
    if (batch <= 0) {
        cudaMemsetAsync(grad, 0, sizeof(float) * kMlpParams, st);
        cudaMemsetAsync(loss, 0, sizeof(float), st);
        return;
    }
    const int tiles = (batch + kTrainRows - 1) / kTrainRows;
    const int blocks = std::min(tiles, kMlpGradBlocks);
    with_arch(arch, [&](auto nin, auto a) {
        auto kernel = k_mlp_train_mma<decltype(nin)::value, decltype(a)::value>;
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
        kernel<<<blocks, kTrainWarps * 32, sizeof(TrainSmem), st>>>(batch, X, T, sel, (const __nv_bfloat16*)wbf,
                                                                    partial);
    });
    const int np = mlp_params(arch);
    k_grad_reduce<<<(np + 1 + 31) / 32, 256, 0, st>>>(blocks, np, partial, grad, loss);
}

void launch_mlp_sample(cudaStream_t st, int batch, uint64_t size, uint64_t seed, uint32_t* sel) {
    if (batch > 0) k_sample<<<grid_of(batch), kBlock, 0, st>>>(batch, size, seed, sel);
}

void launch_adam(cudaStream_t st, int np, float* w, const float* grad, float* m1, float* m2, void* wbf, float lr,
                 int step) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_of(np), kBlock, 0, st>>>(np, w, grad, m1, m2, (__nv_bfloat16*)wbf, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_to_bf16(cudaStream_t st, int np, const float* w, void* wbf) {
    k_to_bf16<<<grid_of(np), kBlock, 0, st>>>(np, w, (__nv_bfloat16*)wbf);
}

void launch_collect(cudaStream_t st, int n, int stride, int offset, uint64_t base, uint64_t cap, const float* feats,
                    const float2* rp, float p_scale, float* X, float* T) {
    const int rows = offset < n ? (n - offset + stride - 1) / stride : 0;
    if (rows > 0) k_collect<<<grid_of(rows), kBlock, 0, st>>>(n, stride, offset, base, cap, feats, rp, p_scale, X, T);
}

}  // namespace psb
