// diag.cu -- FP64 mass, momentum and energy diagnostics.
//
// The state is FP32; these sums are the one place besides the corrector's
// convergence test where FP64 is used. Each block reduces its particles'
// terms in FP64 (warp shuffles, then shared memory) into one partial row;
// a one-block pass then sums the rows in block order. No atomics: the
// result is the same on every run.
//
// Terms per particle i (mass m, interpolated velocity v, position x,
// density rho from the last density pass, gravity g):
//   mass m; momentum m v; kinetic energy m |v|^2 / 2; potential energy
//   -m g.x; |rho - rho0| / rho0 (summed for the mean, and its max).
// No counterpart in the reference, which reports none of them.
#include "psb_internal.cuh"

namespace psb {

namespace {

constexpr int kDiagThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Partial rows over slots [first, first + count): one row of kDiagTerms per block.
__global__ void __launch_bounds__(kDiagThreads) k_diag_partial(int first, int count, double mass, double rho0,
                                                              double gx, double gy, double gz,
                                                              const float4* __restrict__ pos,
                                                              const float4* __restrict__ vel,
                                                              const float2* __restrict__ rp,
                                                              double* __restrict__ rows) {
    __shared__ double s[kDiagThreads / 32][kDiagTerms];
    const int i = blockIdx.x * kDiagThreads + threadIdx.x;
    double t[kDiagTerms] = {};
    if (i < count) {
        const int k = first + i;
        const float4 x = pos[k], v = vel[k];
        const double vx = v.x, vy = v.y, vz = v.z;
        t[0] = mass;
        t[1] = mass * vx; t[2] = mass * vy; t[3] = mass * vz;
        t[4] = 0.5 * mass * (vx * vx + vy * vy + vz * vz);
        t[5] = -mass * (gx * (double)x.x + gy * (double)x.y + gz * (double)x.z);
        const double e = fabs((double)rp[k].x - rho0) / rho0;
        t[6] = e;
        t[7] = e;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kDiagTerms; ++q) {
        const double r = q == 7 ? warp_max(t[q]) : warp_sum(t[q]);
        if (lane == 0) s[warp][q] = r;
    }
    __syncthreads();
    if (threadIdx.x < kDiagTerms) {
        const int q = threadIdx.x;
        double r = s[0][q];
        for (int w = 1; w < kDiagThreads / 32; ++w) r = q == 7 ? fmax(r, s[w][q]) : r + s[w][q];
        rows[(size_t)blockIdx.x * kDiagTerms + q] = r;
    }
}

// Sums nrows partial rows in order into out[0..kDiagTerms).
__global__ void k_diag_final(int nrows, const double* __restrict__ rows, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= kDiagTerms) return;
    double r = 0.0;
    for (int b = 0; b < nrows; ++b) {
        const double v = rows[(size_t)b * kDiagTerms + q];
        r = q == 7 ? fmax(r, v) : r + v;
    }
    out[q] = r;
}

}  // namespace

int diag_rows(int count) { return (count + kDiagThreads - 1) / kDiagThreads; }

void launch_diagnostics(cudaStream_t st, int first, int count, double mass, double rho0, const float g[3],
                        const float4* pos, const float4* vel, const float2* rp, double* rows, double* out) {
    const int nb = diag_rows(count);
    if (nb > 0)
        k_diag_partial<<<nb, kDiagThreads, 0, st>>>(first, count, mass, rho0, g[0], g[1], g[2], pos, vel, rp, rows);
    k_diag_final<<<1, 32, 0, st>>>(nb, rows, out);
}

}  // namespace psb
