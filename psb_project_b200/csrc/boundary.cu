// boundary.cu -- static boundary particles (config profile), after Akinci,
// Ihmsen, Akinci, Solenthaler & Teschner 2012, "Versatile rigid-fluid
// coupling for incompressible SPH".
//
// A solid is sampled by particles b. Each gets the volume-weighted mass
// psi_b = rho0 / sum_k W(x_b - x_k) over the boundary particles (their
// eq. 5), so that the sampling's density, whatever its spacing, stands for a
// full solid. A fluid particle i gains psi_b W_ib in density and the
// pressure term psi_b p_i/rho0^2 gradW_ib (the fluid's own pressure mirrored
// onto the solid); the kernels in sph.cu add both. The reference has no
// counterpart: its obstacles are analytic collision objects
// (src/Kernel/Collision/*), used here only as the box.
//
// The boundary set is sorted once into its own cell ranges over the scene's
// grid; each step, the fluid particles near its bounding box list their
// boundary neighbours (quads, like the fluid lists).
#include "psb_internal.cuh"

namespace psb {

namespace {

inline int blocks_for(int n) { return (n + kBlock - 1) / kBlock; }

__global__ void k_iota(int n, int* __restrict__ a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// Sorted slot t takes the boundary particle vals[t]; cell ranges from the
// sorted keys.
__global__ void k_bnd_gather(int nb, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const float4* __restrict__ raw, float4* __restrict__ sorted, int* __restrict__ ids,
                             uint32_t* __restrict__ cell_start, uint32_t* __restrict__ cell_end) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const int s = (int)vals[t];
    const float4 x = raw[s];
    sorted[t] = make_float4(x.x, x.y, x.z, 0.f);
    ids[t] = s;
    const uint32_t k = keys[t];
    if (t == 0 || keys[t - 1] != k) cell_start[k] = (uint32_t)t;
    if (t == nb - 1 || keys[t + 1] != k) cell_end[k] = (uint32_t)t + 1u;
}

// psi_b / m of sorted boundary slot t, summed in FP64 over the boundary
// particles in its 27 cells that lie within h.
__global__ void k_bnd_psi(Params P, int nb, const uint32_t* __restrict__ keys, const float4* __restrict__ sorted,
                          const uint32_t* __restrict__ cell_start, const uint32_t* __restrict__ cell_end,
                          float* __restrict__ w) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const int nx = P.g.nx, ny = P.g.ny, nz = P.g.nz;
    const float4 xb = sorted[t];
    const uint32_t key = keys[t];
    const int ci = (int)(key % (uint32_t)nx), cj = (int)((key / (uint32_t)nx) % (uint32_t)ny);
    const int ck = (int)(key / ((uint32_t)nx * (uint32_t)ny));
    double s = 0.0;
    for (int k = max(ck - 1, 0); k <= min(ck + 1, nz - 1); ++k)
        for (int j = max(cj - 1, 0); j <= min(cj + 1, ny - 1); ++j) {
            const uint32_t row = (uint32_t)j * (uint32_t)nx + (uint32_t)k * (uint32_t)nx * (uint32_t)ny;
            for (int a = max(ci - 1, 0); a <= min(ci + 1, nx - 1); ++a) {
                const uint32_t lo = cell_start[row + a];
                if (lo == kEmpty) continue;
                const uint32_t hi = cell_end[row + a];
                for (uint32_t q = lo; q < hi; ++q) {
                    const float4 xk = sorted[q];
                    const float dx = xb.x - xk.x, dy = xb.y - xk.y, dz = xb.z - xk.z;
                    const float qq = (dx * dx + dy * dy + dz * dz) * P.inv_h2;
                    if (qq >= 1.f) continue;
                    const double u = 1.0 - (double)qq;
                    s += u * u * u;
                }
            }
        }
    w[t] = (float)(P.rho0_d / ((double)P.k_rho * s));
}

__global__ void k_bnd_set_w(int nb, const float* __restrict__ w, float4* __restrict__ sorted) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb) sorted[t].w = w[t];
}

// Fluid slot t's boundary neighbours, in increasing boundary slot order.
__global__ void __launch_bounds__(kBlock) k_build_bnd_nbr(Params P, const float4* __restrict__ pos,
                                                          const uint32_t* __restrict__ keys,
                                                          const uint32_t* __restrict__ bnd_start,
                                                          const uint32_t* __restrict__ bnd_end, int* __restrict__ counts,
                                                          int* __restrict__ list, int* __restrict__ flags) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 pi = pos[t];
    int cnt = 0;
    if (pi.x >= P.bnd_lo[0] && pi.x <= P.bnd_hi[0] && pi.y >= P.bnd_lo[1] && pi.y <= P.bnd_hi[1] &&
        pi.z >= P.bnd_lo[2] && pi.z <= P.bnd_hi[2]) {
        const int nx = P.g.nx, ny = P.g.ny, nz = P.g.nz, n = P.n;
        const uint32_t key = keys[t];
        const int ci = (int)(key % (uint32_t)nx), cj = (int)((key / (uint32_t)nx) % (uint32_t)ny);
        const int ck = (int)(key / ((uint32_t)nx * (uint32_t)ny));
        const int a0 = max(ci - 1, 0), a1 = min(ci + 1, nx - 1);
        for (int k = max(ck - 1, 0); k <= min(ck + 1, nz - 1); ++k)
            for (int j = max(cj - 1, 0); j <= min(cj + 1, ny - 1); ++j) {
                const uint32_t row = (uint32_t)j * (uint32_t)nx + (uint32_t)k * (uint32_t)nx * (uint32_t)ny;
                uint32_t lo = kEmpty, hi = 0;
                for (int a = a0; a <= a1; ++a) {
                    const uint32_t s = bnd_start[row + a];
                    if (s != kEmpty) {
                        if (lo == kEmpty) lo = s;
                        hi = bnd_end[row + a];
                    }
                }
                if (lo == kEmpty) continue;
                for (uint32_t q = lo; q < hi; ++q) {
                    const float4 xb = P.bnd[q];
                    const float dx = pi.x - xb.x, dy = pi.y - xb.y, dz = pi.z - xb.z;
                    if (dx * dx + dy * dy + dz * dz > P.h2_hi) continue;
                    if (cnt < P.bnd_cap) list[nbr_index(cnt, n, t)] = (int)q;
                    ++cnt;
                }
            }
    }
    counts[t] = cnt;
    if (cnt > P.bnd_cap) atomicOr(&flags[0], 1);
}

// F_b = - sum_j m a_j^b over the fluid particles j within h of the
// boundary particle at xb, a_j^b = k_grad (psi_b / m) pV_j (1-u)^2 x^_jb
// the mirrored-pressure acceleration the boundary particle gives j (sph.cu,
// boundary_pressure); the fluid's cells are walked around xb.
__device__ float3 bnd_reaction_at(const Params& P, float4 xb, const float4* __restrict__ fluid_pos,
                                  const float2* __restrict__ fluid_rp, const uint32_t* __restrict__ cell_start,
                                  const uint32_t* __restrict__ cell_end) {
    const int nx = P.g.nx, ny = P.g.ny, nz = P.g.nz;
    int c[3];
    const float lo[3] = {P.g.gx, P.g.gy, P.g.gz};
    const float x[3] = {xb.x, xb.y, xb.z};
    const int dims[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        const double q = floor(((double)x[a] - (double)lo[a]) / (double)P.g.cell);
        c[a] = q < 0.0 ? 0 : (q >= (double)dims[a] ? dims[a] - 1 : (int)q);
    }
    const float ir0 = 1.f / (P.rho0 * P.rho0);
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = max(c[2] - 1, 0); k <= min(c[2] + 1, nz - 1); ++k)
        for (int j = max(c[1] - 1, 0); j <= min(c[1] + 1, ny - 1); ++j) {
            const uint32_t row = (uint32_t)j * (uint32_t)nx + (uint32_t)k * (uint32_t)nx * (uint32_t)ny;
            for (int a = max(c[0] - 1, 0); a <= min(c[0] + 1, nx - 1); ++a) {
                const uint32_t q0 = cell_start[row + a];
                if (q0 == kEmpty) continue;
                const uint32_t q1 = cell_end[row + a];
                for (uint32_t q = q0; q < q1; ++q) {
                    const float4 xj = fluid_pos[q];
                    const float dx = xj.x - xb.x, dy = xj.y - xb.y, dz = xj.z - xb.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (!(r2 > 0.f) || r2 * P.inv_h2 >= 1.f) continue;
                    const float rinv = rsqrtf(r2);
                    const float om = 1.f - r2 * rinv * P.inv_h;
                    const float w = fluid_rp[q].y * ir0 * om * om * rinv;
                    s.x += w * dx; s.y += w * dy; s.z += w * dz;
                }
            }
        }
    const float k = -P.mass * P.k_grad * xb.w;
    return make_float3(k * s.x, k * s.y, k * s.z);
}

// Boundary slot b's reaction at the fluid's state.
__global__ void __launch_bounds__(kBlock) k_bnd_reaction(Params P, int nb, const float4* __restrict__ fluid_pos,
                                                         const float2* __restrict__ fluid_rp,
                                                         const uint32_t* __restrict__ cell_start,
                                                         const uint32_t* __restrict__ cell_end,
                                                         float4* __restrict__ force) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const float3 F = bnd_reaction_at(P, P.bnd[b], fluid_pos, fluid_rp, cell_start, cell_end);
    force[b] = make_float4(F.x, F.y, F.z, 0.f);
}

// Moving boundary: the reaction at the committed pressures of the current
// correction (the fluid at the step's start positions, as the config
// pressure force) and the boundary's prediction with it. The velocity and
// position updates are the DEM step's (v += (f + F) / m dt, x += v dt), so
// the spheres' next positions are the last prediction's wherever no wall
// projects them.
__global__ void __launch_bounds__(kBlock) k_bnd_move(Params P, int nb, const float4* __restrict__ fluid_pos,
                                                     const float2* __restrict__ fluid_rp,
                                                     const uint32_t* __restrict__ cell_start,
                                                     const uint32_t* __restrict__ cell_end,
                                                     const float4* __restrict__ vel, const float4* __restrict__ fext,
                                                     float inv_mass, float4* __restrict__ pred,
                                                     float4* __restrict__ force) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const float4 xb = P.bnd[b];
    const float3 F = bnd_reaction_at(P, xb, fluid_pos, fluid_rp, cell_start, cell_end);
    const float4 v0 = vel[b], f = fext[b];
    const float vx = v0.x + (f.x + F.x) * inv_mass * P.dt;
    const float vy = v0.y + (f.y + F.y) * inv_mass * P.dt;
    const float vz = v0.z + (f.z + F.z) * inv_mass * P.dt;
    pred[b] = make_float4(xb.x + vx * P.dt, xb.y + vy * P.dt, xb.z + vz * P.dt, xb.w);
    force[b] = make_float4(F.x, F.y, F.z, 0.f);
}

__global__ void k_gather4(int nb, const int* __restrict__ ids, const float4* __restrict__ src,
                          float4* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb) dst[t] = src[ids[t]];
}

}  // namespace

void launch_bnd_move(cudaStream_t st, const Params& P, int nb, const float4* fluid_pos, const float2* fluid_rp,
                     const uint32_t* cell_start, const uint32_t* cell_end, const float4* vel, const float4* fext,
                     float inv_mass, float4* pred, float4* force) {
    if (nb > 0)
        k_bnd_move<<<blocks_for(nb), kBlock, 0, st>>>(P, nb, fluid_pos, fluid_rp, cell_start, cell_end, vel, fext,
                                                      inv_mass, pred, force);
}

void launch_bnd_gather4(cudaStream_t st, int nb, const int* ids, const float4* src, float4* dst) {
    if (nb > 0) k_gather4<<<blocks_for(nb), kBlock, 0, st>>>(nb, ids, src, dst);
}

void launch_bnd_reaction(cudaStream_t st, const Params& P, int nb, const float4* fluid_pos, const float2* fluid_rp,
                         const uint32_t* cell_start, const uint32_t* cell_end, float4* force) {
    if (nb > 0)
        k_bnd_reaction<<<blocks_for(nb), kBlock, 0, st>>>(P, nb, fluid_pos, fluid_rp, cell_start, cell_end, force);
}

int launch_bnd_prepare(cudaStream_t st, const Params& P, int nb, const float4* raw, int* iota, uint32_t* keys[2],
                       uint32_t* vals[2], uint32_t* hist, int hist_blocks, int key_bits, float4* sorted, int* ids,
                       float* w, uint32_t* cell_start, uint32_t* cell_end, int* clamped) {
    if (nb <= 0) return 0;
    Params Q = P;
    Q.n = nb;
    Q.scenes = nullptr;
    k_iota<<<blocks_for(nb), kBlock, 0, st>>>(nb, iota);
    launch_cell_keys(st, Q, raw, iota, keys[0], vals[0], clamped);
    const int res = radix_sort(st, nb, key_bits, keys, vals, hist, hist_blocks);
    k_bnd_gather<<<blocks_for(nb), kBlock, 0, st>>>(nb, keys[res], vals[res], raw, sorted, ids, cell_start, cell_end);
    k_bnd_psi<<<blocks_for(nb), kBlock, 0, st>>>(Q, nb, keys[res], sorted, cell_start, cell_end, w);
    k_bnd_set_w<<<blocks_for(nb), kBlock, 0, st>>>(nb, w, sorted);
    return res;
}

void launch_build_bnd_nbr(cudaStream_t st, const Params& P, const float4* pos, const uint32_t* keys,
                          const uint32_t* bnd_start, const uint32_t* bnd_end, int* counts, int* list, int* flags) {
    if (P.n > 0)
        k_build_bnd_nbr<<<blocks_for(P.n), kBlock, 0, st>>>(P, pos, keys, bnd_start, bnd_end, counts, list, flags);
}

}  // namespace psb
