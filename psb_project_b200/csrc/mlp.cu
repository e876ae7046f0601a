// mlp.cu -- learned pressure warm start for the PCISPH corrector.
//
// A per-particle MLP, 7 -> 64 -> 64 -> 1 with ReLU, predicts each step's
// initial pressure so that the eta-controlled corrector (unchanged; it still
// iterates to the same eta and decides convergence) starts closer to the
// converged pressure. The reference has no counterpart: it starts every
// step from p = 0 (PciSphSystem_Kernel.cu:131).
//
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
// Training is on the GPU: (features, converged pressure) pairs are collected
// from steps of the same eta-loop, then minibatch Adam on an MSE loss, with a
// fused forward/backward kernel whose weight gradients are reduced per warp
// with shuffles before one atomic add per warp.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "psb_internal.cuh"

namespace psb {

namespace {

constexpr int kIn = 7, kH = 64;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
static_assert(oB3 + 1 == kMlpParams, "parameter layout");

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// ReLU: exact, and free of the special-function unit (a SiLU's exponential
// and reciprocal bounded the inference kernel)
__device__ __forceinline__ float act(float z) { return fmaxf(z, 0.f); }
__device__ __forceinline__ float act_grad(float z) { return z > 0.f ? 1.f : 0.f; }

// ---- inference -----------------------------------------------------------------
// Tensor-core inference: one warp evaluates 16 particles per pass with
// mma.sync.m16n8k16 (BF16 inputs, FP32 accumulation). Layer 1 is a
// [16 x 16] x [16 x 64] product (7 inputs, 9 zero pads), layer 2
// [16 x 64] x [64 x 64]; the layer-1 accumulator fragments, rounded to BF16,
// are exactly the A fragments of layer 2 (rows groupID and groupID + 8,
// columns 2 tig + {0, 1} of each 8-wide tile). The output layer (64 -> 1) is
// a per-thread dot product finished with two shuffles.
// Shared memory: W1 and W2 as BF16 pairs, rows padded to 36 words so that
// the eight groups of a B-fragment load fall in distinct banks.
constexpr int kW2Stride = 36;     // 32-bit words per padded 64-wide row
constexpr int kW1Stride = 4;      // 8 BF16 per row (7 used)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}


// y_raw != nullptr: write the raw output y there (host-facing evaluation)
// instead of the initial pressure max(0, y) p_scale into rp.
__global__ void __launch_bounds__(256) k_mlp_infer_mma(int n, const float* __restrict__ feats,
                                                       const __nv_bfloat16* __restrict__ w, float p_scale,
                                                       float2* __restrict__ rp, float* __restrict__ y_raw) {
    __shared__ uint32_t sW1[kH * kW1Stride];
    __shared__ uint32_t sW2[kH * kW2Stride];
    __shared__ float sB1[kH], sB2[kH], sW3[kH];
    __shared__ float sB3;
    for (int i = threadIdx.x; i < kH * kW1Stride; i += blockDim.x) {
        const int r = i / kW1Stride, k = 2 * (i % kW1Stride);
        const float lo = k < kIn ? __bfloat162float(w[oW1 + r * kIn + k]) : 0.f;
        const float hi = k + 1 < kIn ? __bfloat162float(w[oW1 + r * kIn + k + 1]) : 0.f;
        sW1[i] = pack_bf16(lo, hi);
    }
    for (int i = threadIdx.x; i < kH * 32; i += blockDim.x) {
        const int r = i / 32, k = 2 * (i % 32);
        sW2[r * kW2Stride + i % 32] =
            pack_bf16(__bfloat162float(w[oW2 + r * kH + k]), __bfloat162float(w[oW2 + r * kH + k + 1]));
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        sB1[i] = __bfloat162float(w[oB1 + i]);
        sB2[i] = __bfloat162float(w[oB2 + i]);
        sW3[i] = __bfloat162float(w[oW3 + i]);
    }
    if (threadIdx.x == 0) sB3 = __bfloat162float(w[oB3]);
    __syncthreads();

    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    for (int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n; tile += warps_total) {
        const int r0 = tile * 16 + gid, r1 = r0 + 8;
        // layer 1: A = features (cols 0..6 real)
        uint32_t a0 = 0u, a1 = 0u;
        {
            const int k = 2 * tig;
            if (k < kIn) {
                const float f00 = r0 < n ? feats[(size_t)r0 * 8 + k] : 0.f;
                const float f01 = r0 < n ? feats[(size_t)r0 * 8 + k + 1] : 0.f;
                const float f10 = r1 < n ? feats[(size_t)r1 * 8 + k] : 0.f;
                const float f11 = r1 < n ? feats[(size_t)r1 * 8 + k + 1] : 0.f;
                a0 = pack_bf16(f00, k + 1 < kIn ? f01 : 0.f);
                a1 = pack_bf16(f10, k + 1 < kIn ? f11 : 0.f);
            }
        }
        float z1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int col = nt * 8 + 2 * tig;
            z1[nt][0] = sB1[col]; z1[nt][1] = sB1[col + 1];
            z1[nt][2] = sB1[col]; z1[nt][3] = sB1[col + 1];
            const uint32_t b0 = sW1[(nt * 8 + gid) * kW1Stride + tig];   // k = 2 tig .. 2 tig + 1
            mma_bf16(z1[nt], a0, a1, 0u, 0u, b0, 0u);
        }
        // layer 2: A fragments from layer 1's accumulators
        uint32_t h1[4][4];
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            h1[ks][0] = pack_bf16(act(z1[2 * ks][0]), act(z1[2 * ks][1]));
            h1[ks][1] = pack_bf16(act(z1[2 * ks][2]), act(z1[2 * ks][3]));
            h1[ks][2] = pack_bf16(act(z1[2 * ks + 1][0]), act(z1[2 * ks + 1][1]));
            h1[ks][3] = pack_bf16(act(z1[2 * ks + 1][2]), act(z1[2 * ks + 1][3]));
        }
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int col = nt * 8 + 2 * tig;
            float c[4] = {sB2[col], sB2[col + 1], sB2[col], sB2[col + 1]};
            const uint32_t* wrow = sW2 + (nt * 8 + gid) * kW2Stride;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
                mma_bf16(c, h1[ks][0], h1[ks][1], h1[ks][2], h1[ks][3], wrow[8 * ks + tig], wrow[8 * ks + 4 + tig]);
            // output layer on the BF16-rounded activations
            const float w30 = sW3[col], w31 = sW3[col + 1];
            y0 = fmaf(w30, bf(act(c[0])), y0);
            y0 = fmaf(w31, bf(act(c[1])), y0);
            y1 = fmaf(w30, bf(act(c[2])), y1);
            y1 = fmaf(w31, bf(act(c[3])), y1);
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
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One thread per sample: forward (activations kept in registers, the second
// layer recomputed per unit), MSE loss, backward. Weight gradients are summed
// over the warp with shuffles and added to `grad` once per warp.
// Sample b of the batch is row sel[b] of (X, T) (X stride 8, features 0..6).
__global__ void __launch_bounds__(128) k_mlp_train(int batch, const float* __restrict__ X, const float* __restrict__ T,
                                                   const uint32_t* __restrict__ sel,
                                                   const __nv_bfloat16* __restrict__ w, float* __restrict__ grad,
                                                   float* __restrict__ loss) {
    __shared__ float sw[kMlpParams];
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = b < batch;
    const uint32_t row = valid ? (sel ? sel[b] : (uint32_t)b) : 0u;
    const float inv_b = 1.f / (float)batch;
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[k] = valid ? bf(X[(size_t)row * 8 + k]) : 0.f;
    float h1[kH];
#pragma unroll
    for (int j = 0; j < kH; ++j) {
        float z = sw[oB1 + j];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = fmaf(sw[oW1 + j * kIn + k], x[k], z);
        h1[j] = bf(act(z));
    }
    float y = sw[oB3];
    for (int j = 0; j < kH; ++j) {
        float z = sw[oB2 + j];
#pragma unroll
        for (int k = 0; k < kH; ++k) z = fmaf(sw[oW2 + j * kH + k], h1[k], z);
        y = fmaf(sw[oW3 + j], bf(act(z)), y);
    }
    const float e = valid ? y - T[row] : 0.f;
    const float dy = 2.f * e * inv_b;                     // d(mean e^2)/dy
    const float ls = warp_sum(e * e * inv_b);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, ls);
    const float gb3 = warp_sum(dy);
    if ((threadIdx.x & 31) == 0) atomicAdd(&grad[oB3], gb3);
    float dh1[kH];
#pragma unroll
    for (int k = 0; k < kH; ++k) dh1[k] = 0.f;
    for (int j = 0; j < kH; ++j) {
        float z = sw[oB2 + j];
#pragma unroll
        for (int k = 0; k < kH; ++k) z = fmaf(sw[oW2 + j * kH + k], h1[k], z);
        const float h2 = bf(act(z));
        const float dz2 = dy * sw[oW3 + j] * act_grad(z);
        const float g3 = warp_sum(dy * h2);
        const float g2b = warp_sum(dz2);
        if ((threadIdx.x & 31) == 0) { atomicAdd(&grad[oW3 + j], g3); atomicAdd(&grad[oB2 + j], g2b); }
#pragma unroll
        for (int k = 0; k < kH; ++k) {
            dh1[k] = fmaf(sw[oW2 + j * kH + k], dz2, dh1[k]);
            const float g = warp_sum(dz2 * h1[k]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&grad[oW2 + j * kH + k], g);
        }
    }
#pragma unroll
    for (int j = 0; j < kH; ++j) {
        float z = sw[oB1 + j];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = fmaf(sw[oW1 + j * kIn + k], x[k], z);
        const float dz1 = dh1[j] * act_grad(z);
        const float g1b = warp_sum(dz1);
        if ((threadIdx.x & 31) == 0) atomicAdd(&grad[oB1 + j], g1b);
#pragma unroll
        for (int k = 0; k < kIn; ++k) {
            const float g = warp_sum(dz1 * x[k]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&grad[oW1 + j * kIn + k], g);
        }
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

}  // namespace

void launch_zero_pressure(cudaStream_t st, int n, float2* rp) {
    if (n > 0) k_zero_pressure<<<grid_of(n), kBlock, 0, st>>>(n, rp);
}


void launch_mlp_infer(cudaStream_t st, int n, const float* feats, const void* wbf, float p_scale, float2* rp) {
    if (n <= 0) return;
    const int tiles = (n + 15) / 16;
    const int blocks = std::min((tiles + 7) / 8, 148 * 8);      // 8 warps per block, grid-stride over tiles
    k_mlp_infer_mma<<<blocks, 256, 0, st>>>(n, feats, (const __nv_bfloat16*)wbf, p_scale, rp, nullptr);
}


// Host-facing forward through the tensor-core kernel the warm start uses
// (rows of stride 8).
void launch_mlp_forward(cudaStream_t st, int n, const float* X, int stride, const void* wbf, float* y) {
    if (n <= 0) return;
    (void)stride;
    const int tiles = (n + 15) / 16;
    const int blocks = std::min((tiles + 7) / 8, 148 * 8);
    k_mlp_infer_mma<<<blocks, 256, 0, st>>>(n, X, (const __nv_bfloat16*)wbf, 1.f, nullptr, y);
}

void launch_mlp_grad(cudaStream_t st, int batch, const float* X, const float* T, const uint32_t* sel, const void* wbf,
                     float* grad, float* loss) {
    cudaMemsetAsync(grad, 0, sizeof(float) * kMlpParams, st);
    cudaMemsetAsync(loss, 0, sizeof(float), st);
    if (batch > 0) k_mlp_train<<<grid_of(batch, 128), 128, 0, st>>>(batch, X, T, sel, (const __nv_bfloat16*)wbf, grad, loss);
}

void launch_mlp_sample(cudaStream_t st, int batch, uint64_t size, uint64_t seed, uint32_t* sel) {
    if (batch > 0) k_sample<<<grid_of(batch), kBlock, 0, st>>>(batch, size, seed, sel);
}

void launch_adam(cudaStream_t st, float* w, const float* grad, float* m1, float* m2, void* wbf, float lr, int step) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_of(kMlpParams), kBlock, 0, st>>>(kMlpParams, w, grad, m1, m2, (__nv_bfloat16*)wbf, lr, b1, b2, 1e-8f,
                                                   c1, c2);
}

void launch_to_bf16(cudaStream_t st, const float* w, void* wbf) {
    k_to_bf16<<<grid_of(kMlpParams), kBlock, 0, st>>>(kMlpParams, w, (__nv_bfloat16*)wbf);
}

void launch_collect(cudaStream_t st, int n, int stride, int offset, uint64_t base, uint64_t cap, const float* feats,
                    const float2* rp, float p_scale, float* X, float* T) {
    const int rows = offset < n ? (n - offset + stride - 1) / stride : 0;
    if (rows > 0) k_collect<<<grid_of(rows), kBlock, 0, st>>>(n, stride, offset, base, cap, feats, rp, p_scale, X, T);
}

}  // namespace psb
