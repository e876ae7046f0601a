// compat.cu -- the reference's extern "C" launchers (include/psb_compat.h)
// on the reference's own device layouts, so its system classes link
// unchanged against libpsb.so.
//
// The grid, integration, contact and wall launchers are elementwise or
// per-particle list walks on the caller's AoS double3 buffers, in FP64 with
// the reference's expression order (its double3 operator/ multiplies by the
// reciprocal; dt reaches the kernels as float). pci_SPH_update runs the
// B200 step itself (reference profile) on a context kept per process.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "psb.h"
#include "psb_compat.h"
#include "psb_internal.cuh"

namespace {

constexpr int kT = 256;
inline unsigned nblocks(long long n) { return (unsigned)((n + kT - 1) / kT); }

__device__ int g_compat_overflow;     // set when a cell or a neighbour list is full

__device__ __forceinline__ double3 ld3(const double* a, long long i) {
    return make_double3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
}
__device__ __forceinline__ void st3(double* a, long long i, double3 v) {
    a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z;
}

__global__ void k_create_cells(double xC, double yC, double zC, double l, double w, double d, float cell, int nx, int ny,
                               int nz, double3* centres, int* counts) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)nx * ny * nz) return;
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    counts[c] = 0;
    centres[c] = make_double3(xC - (l / 2) + (cell / 2) + i * cell, yC - (w / 2) + (cell / 2) + j * cell,
                              zC - (d / 2) + (cell / 2) + k * cell);
}

__device__ __forceinline__ bool cell_of(const double* pos, long long p, float3 Min, float cell, int nx, int ny, int nz,
                                        int& i, int& j, int& k) {
    i = (int)floor((pos[3 * p] - Min.x) / cell);
    j = (int)floor((pos[3 * p + 1] - Min.y) / cell);
    k = (int)floor((pos[3 * p + 2] - Min.z) / cell);
    return i >= 0 && j >= 0 && k >= 0 && i < nx && j < ny && k < nz;
}

__global__ void k_store(const double* pos, unsigned n, int* counts, int* slots, float3 Min, float cell, int nx, int ny,
                        int nz) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int i, j, k;
    if (!cell_of(pos, p, Min, cell, nx, ny, nz, i, j, k)) { g_compat_overflow = 1; return; }
    const long long c = i + (long long)j * nx + (long long)k * nx * ny;
    const int s = atomicAdd(&counts[c], 1);
    if (s < PSB_COMPAT_MAXPARTICLES) slots[c * PSB_COMPAT_MAXPARTICLES + s] = (int)p;
    else g_compat_overflow = 1;
}

__global__ void k_search(const double* pos, const double* radius, const int* slots, const int* counts, int nx, int ny,
                         int nz, float cell, float3 Min, double scale, int* nbr_n, int* nbr, unsigned n) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int cnt = 0;
    int I, J, K;
    if (cell_of(pos, p, Min, cell, nx, ny, nz, I, J, K)) {
        const int r = (int)ceil(scale);
        const double3 x = ld3(pos, p);
        for (int i = I - r; i <= I + r; ++i)
            for (int j = J - r; j <= J + r; ++j)
                for (int k = K - r; k <= K + r; ++k) {
                    if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
                    const long long c = i + (long long)j * nx + (long long)k * nx * ny;
                    const int m = min(counts[c], PSB_COMPAT_MAXPARTICLES);
                    for (int s = 0; s < m; ++s) {
                        const int q = slots[c * PSB_COMPAT_MAXPARTICLES + s];
                        const double dx = x.x - pos[3 * (long long)q], dy = x.y - pos[3 * (long long)q + 1],
                                     dz = x.z - pos[3 * (long long)q + 2];
                        const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                                        __dmul_rn(dz, dz)));
                        if (d <= radius[p]) {
                            if (cnt < PSB_COMPAT_MAX_NEIGHBOURS) nbr[p * PSB_COMPAT_MAX_NEIGHBOURS + cnt] = q;
                            else g_compat_overflow = 1;
                            ++cnt;
                        }
                    }
                }
    }
    nbr_n[p] = min(cnt, PSB_COMPAT_MAX_NEIGHBOURS);
}

__global__ void k_leapfrog(double* vav, double* vap, double* xold, double* x, const double* f, const double* rho, float dt,
                           int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double3 v = ld3(vap, i);
    st3(vav, i, v);
    const double ir = 1.0 / rho[i];
    const double3 F = ld3(f, i);
    const double3 vn = make_double3(v.x + (F.x * ir) * dt, v.y + (F.y * ir) * dt, v.z + (F.z * ir) * dt);
    st3(vap, i, vn);
    const double3 p = ld3(x, i);
    st3(xold, i, p);
    st3(x, i, make_double3(p.x + vn.x * dt, p.y + vn.y * dt, p.z + vn.z * dt));
}

__global__ void k_interp(const double* vav, const double* vap, double* vold, double* v, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st3(vold, i, ld3(v, i));
    const double3 a = ld3(vav, i), b = ld3(vap, i);
    st3(v, i, make_double3((a.x + b.x) * 0.5, (a.y + b.y) * 0.5, (a.z + b.z) * 0.5));
}

__global__ void k_euler(double* x, double* v, const double* f, const double* mass, float dt, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double3 v0 = ld3(v, i), F = ld3(f, i);
    const double im = 1.0 / mass[i];
    st3(v, i, make_double3(v0.x + (F.x * im) * dt, v0.y + (F.y * im) * dt, v0.z + (F.z * im) * dt));
    const double3 p = ld3(x, i);
    st3(x, i, make_double3(p.x + v0.x * dt, p.y + v0.y * dt, p.z + v0.z * dt));
}

__global__ void k_contacts(const double* x, double* f, const double* radius, const double* spring, const int* nbr_n,
                           const int* nbr, int n) {
    const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const double3 xa = ld3(x, a);
    double3 F = ld3(f, a);
    const int m = nbr_n[a];
    for (int s = 0; s < m; ++s) {
        const int b = nbr[a * PSB_COMPAT_MAX_NEIGHBOURS + s];
        const double rx = x[3 * (long long)b] - xa.x, ry = x[3 * (long long)b + 1] - xa.y, rz = x[3 * (long long)b + 2] - xa.z;
        const double dist = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)));
        if (!(dist > 0)) continue;
        const float R = (float)(radius[a] + radius[b]);
        if (!(dist < R * 2.0f)) continue;
        const double inv = 1.0 / dist;
        const double s_ = -spring[a] * ((double)R - dist);
        F.x = F.x + s_ * (rx * inv);
        F.y = F.y + s_ * (ry * inv);
        F.z = F.z + s_ * (rz * inv);
    }
    st3(f, a, F);
}

__global__ void k_box(double* x, double* v, float3 Min, float3 Max, float r, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double3 p = ld3(x, i);
    double3 pI = p, nI = make_double3(0, 0, 0);
    if (p.x >= Max.x - r) { pI.x = Max.x - r; nI.x = -1.0; }
    if (p.y >= Max.y - r) { pI.y = Max.y - r; nI.y = -1.0; }
    if (p.z >= Max.z - r) { pI.z = Max.z - r; nI.z = -1.0; }
    if (p.x <= Min.x + r) { pI.x = Min.x + r; nI.x = 1.0; }
    if (p.y <= Min.y + r) { pI.y = Min.y + r; nI.y = 1.0; }
    if (p.z <= Min.z + r) { pI.z = Min.z + r; nI.z = 1.0; }
    const double l = sqrt(nI.x * nI.x + nI.y * nI.y + nI.z * nI.z);
    if (l > 0) {
        nI = make_double3(nI.x / l, nI.y / l, nI.z / l);
        const double3 u = ld3(v, i);
        const double vd = u.x * nI.x + u.y * nI.y + u.z * nI.z;
        st3(x, i, pI);
        st3(v, i, make_double3(u.x - vd * nI.x, u.y - vd * nI.y, u.z - vd * nI.z));
    }
}

// bounding box of AoS double positions as ordered integers of the float
// coordinates rounded outward
__device__ __forceinline__ unsigned ord(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__global__ void k_bbox(const double* x, int n, unsigned* lo_hi) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = 0; a < 3; ++a) {
        const double c = x[3 * i + a];
        atomicMin(&lo_hi[a], ord(__double2float_rd(c)));
        atomicMax(&lo_hi[3 + a], ord(__double2float_ru(c)));
    }
}

__global__ void k_copy_f32_to_f64(const float* s, double* d, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = (double)s[i];
}

void report_overflow(const char* where) {
    int f = 0;
    cudaMemcpyFromSymbol(&f, g_compat_overflow, sizeof(int));
    if (f) {
        std::fprintf(stderr, "%s: a particle left the grid, a cell held more than %d particles or a list more "
                             "than %d neighbours (clamped)\n", where, PSB_COMPAT_MAXPARTICLES, PSB_COMPAT_MAX_NEIGHBOURS);
        const int z = 0;
        cudaMemcpyToSymbol(g_compat_overflow, &z, sizeof(int));
    }
}

// ---- pci_SPH_update: the B200 step on a per-process context ------------------------
struct PciContext {
    psb_ctx* ctx = nullptr;
    psb_scene sc{};
    int device = -1;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    unsigned* bbox = nullptr;
    float* stage = nullptr;
    int stage_n = 0;
};
PciContext g_pci;

bool same_params(const psb_scene& a, const psb_scene& b) {
    return a.h == b.h && a.mass == b.mass && a.rho0 == b.rho0 && a.k == b.k && a.mu == b.mu && a.sigma == b.sigma &&
           a.l == b.l && a.dt == b.dt;
}

}  // namespace

extern "C" {

void createGrid(double xC, double yC, double zC, double length, double width, double depth, float sizeCell,
                UniformGrid* grid) {
    grid->Min.x = xC - length / 2; grid->Min.y = yC - width / 2; grid->Min.z = zC - depth / 2;
    grid->Max.x = xC + length / 2; grid->Max.y = yC + width / 2; grid->Max.z = zC + depth / 2;
    grid->nbCellsX = (int)ceil(length / sizeCell);
    grid->nbCellsY = (int)ceil(width / sizeCell);
    grid->nbCellsZ = (int)ceil(depth / sizeCell);
    grid->sizeCell = sizeCell;
    const long long nx = grid->nbCellsX, ny = grid->nbCellsY, nz = grid->nbCellsZ;
    const long long size = nx + nx * ny + nz * ny * nx;   // the reference's allocation (UniformGrid.cu:33-35)
    cudaMalloc((void**)&grid->m_dPos, sizeof(double3) * size);
    cudaMalloc((void**)&grid->indexParticles, sizeof(int) * PSB_COMPAT_MAXPARTICLES * size);
    cudaMalloc((void**)&grid->nbParticles, sizeof(int) * size);
    cudaMemset(grid->nbParticles, 0, sizeof(int) * size);
    k_create_cells<<<nblocks(nx * ny * nz), kT>>>(xC, yC, zC, length, width, depth, sizeCell, (int)nx, (int)ny, (int)nz,
                                                  grid->m_dPos, grid->nbParticles);
    cudaDeviceSynchronize();
}

void _finalizeGrid(UniformGrid* grid) {
    delete[] grid->m_hPos;
    delete[] grid->m_hIsoVal;
    cudaFree(grid->m_dPos);
    cudaFree(grid->nbParticles);
    cudaFree(grid->indexParticles);
    cudaFree(grid->m_dIsoVal);
}

void reinitCells(UniformGrid* grid) {
    cudaMemset(grid->nbParticles, 0, sizeof(int) * (size_t)grid->nbCellsX * grid->nbCellsY * grid->nbCellsZ);
    cudaDeviceSynchronize();
}

void storeParticles(UniformGrid* grid, double* pos, unsigned int nbBodies) {
    if (nbBodies) {
        k_store<<<nblocks(nbBodies), kT>>>(pos, nbBodies, grid->nbParticles, grid->indexParticles, grid->Min,
                                           grid->sizeCell, grid->nbCellsX, grid->nbCellsY, grid->nbCellsZ);
        cudaDeviceSynchronize();
    }
    report_overflow("storeParticles");
}

void searchNeighbooring(double* pos, double* radius, UniformGrid* grid, double scale, partVoisine voisines,
                        unsigned int nbBodies) {
    if (nbBodies) {
        k_search<<<nblocks(nbBodies), kT>>>(pos, radius, grid->indexParticles, grid->nbParticles, grid->nbCellsX,
                                            grid->nbCellsY, grid->nbCellsZ, grid->sizeCell, grid->Min, scale,
                                            voisines.nbVoisines, voisines.listeVoisine, nbBodies);
        cudaDeviceSynchronize();
    }
    report_overflow("searchNeighbooring");
}

void integrateSPHSystem(double* velInterAv, double* velInterAp, double* oldPos, double* newPos, double* forces,
                        double* densities, double dt, int numBodies) {
    if (numBodies <= 0) return;
    k_leapfrog<<<nblocks(numBodies), kT>>>(velInterAv, velInterAp, oldPos, newPos, forces, densities, (float)dt,
                                           numBodies);
    cudaDeviceSynchronize();
}

void interpolateSPHVelocities(double* velInterAv, double* velInterAp, double* oldVel, double* newVel, int numBodies) {
    if (numBodies <= 0) return;
    k_interp<<<nblocks(numBodies), kT>>>(velInterAv, velInterAp, oldVel, newVel, numBodies);
    cudaDeviceSynchronize();
}

void integrateSystem(double* oldPos, double* newPos, double* oldVel, double* newVel, double* forces, double* mass,
                     double dt, int start, int numBodies) {
    (void)oldPos; (void)oldVel; (void)start;    // integrateSystem reads neither (System.cu:6-12)
    if (numBodies <= 0) return;
    k_euler<<<nblocks(numBodies), kT>>>(newPos, newVel, forces, mass, (float)dt, numBodies);
    cudaDeviceSynchronize();
}

void interactionSystem(double* oldPos, double* oldVel, double* forces, double* interactionRadius, double* spring,
                       double* damping, double* shear, double* attraction, partVoisine voisines, int numBodies) {
    (void)oldVel; (void)damping; (void)shear; (void)attraction;
    if (numBodies <= 0) return;
    k_contacts<<<nblocks(numBodies), kT>>>(oldPos, forces, interactionRadius, spring, voisines.nbVoisines,
                                           voisines.listeVoisine, numBodies);
    cudaDeviceSynchronize();
}

void collisionSystem_Box_CUDA(double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                              int nbBodiesP, psb_vec3 Min, psb_vec3 Max, bool container, float elast) {
    (void)oldVel; (void)dt; (void)container; (void)elast;   // the restitution term is commented out there
    if (nbBodiesP <= 0) return;
    const float3 mn = make_float3((float)Min.e[0], (float)Min.e[1], (float)Min.e[2]);
    const float3 mx = make_float3((float)Max.e[0], (float)Max.e[1], (float)Max.e[2]);
    k_box<<<nblocks(nbBodiesP), kT>>>(newPos, newVel, mn, mx, radiusParticle, nbBodiesP);
    cudaDeviceSynchronize();
}

void pci_SPH_update(double* oldPos, double* pos, double* vel, double* velInterAv, double* velInterAp,
                    double* restore_oldPos, double* restore_pos, double* restore_velInterAv,
                    double* restore_velInterAp, double* mass, double* radius, double* density, double* restDensity,
                    double* densityError, double* pressure, double* k, double* viscosity, double* l,
                    double* surfaceTension, double threshold, partVoisine voisines, double* normales,
                    double* forceViscosity, double* forceSurface, double* forcePressure, double* forceAccum, float dt,
                    unsigned int nbBodies) {
    (void)restore_oldPos; (void)restore_pos; (void)restore_velInterAv; (void)restore_velInterAp; (void)densityError;
    (void)threshold; (void)voisines; (void)normales; (void)forceViscosity; (void)forceSurface; (void)forcePressure;
    (void)forceAccum;
    if (nbBodies == 0) return;
    const int n = (int)nbBodies;
    cudaDeviceSynchronize();
    int dev = 0;
    cudaGetDevice(&dev);
    double p0[7];
    const double* src[7] = {mass, radius, restDensity, k, viscosity, l, surfaceTension};
    for (int i = 0; i < 7; ++i) cudaMemcpy(&p0[i], src[i], sizeof(double), cudaMemcpyDeviceToHost);
    if (!g_pci.bbox || g_pci.device != dev) cudaMalloc((void**)&g_pci.bbox, 6 * sizeof(unsigned));
    const unsigned init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    cudaMemcpy(g_pci.bbox, init, sizeof(init), cudaMemcpyHostToDevice);
    k_bbox<<<nblocks(n), kT>>>(pos, n, g_pci.bbox);
    unsigned bb[6];
    cudaMemcpy(bb, g_pci.bbox, sizeof(bb), cudaMemcpyDeviceToHost);
    auto unord_h = [](unsigned u) { u = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u; float f; std::memcpy(&f, &u, 4); return f; };
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = unord_h(bb[a]); hi[a] = unord_h(bb[3 + a]); }

    psb_scene s{};
    s.h = p0[1]; s.mass = p0[0]; s.rho0 = p0[2]; s.k = p0[3]; s.mu = p0[4]; s.l = p0[5]; s.sigma = p0[6];
    s.dt = dt;
    const bool fits = g_pci.ctx && g_pci.device == dev && same_params(s, g_pci.sc) && n <= g_pci.sc.n_max &&
                      lo[0] >= g_pci.lo[0] && lo[1] >= g_pci.lo[1] && lo[2] >= g_pci.lo[2] &&
                      hi[0] <= g_pci.hi[0] && hi[1] <= g_pci.hi[1] && hi[2] <= g_pci.hi[2];
    if (!fits) {
        if (g_pci.ctx) psb_destroy(g_pci.ctx);
        g_pci.ctx = nullptr;
        const float cell = (float)s.h;      // createGrid(..., h): the reference's cell
        for (int a = 0; a < 3; ++a) {
            const float ext = hi[a] - lo[a];
            g_pci.lo[a] = lo[a] - 0.25f * ext - 2.f * cell;
            g_pci.hi[a] = hi[a] + 0.25f * ext + 2.f * cell;
            s.grid_min[a] = g_pci.lo[a] - cell;
            s.dims[a] = (int)std::ceil((g_pci.hi[a] - g_pci.lo[a]) / cell) + 2;
            s.box_min[a] = -1e6f;      // pci_SPH_update has no walls (the class collides afterwards)
            s.box_max[a] = 1e6f;
        }
        s.cell = cell;
        s.n_max = n + n / 4 + 1;
        s.profile = PSB_PROFILE_REF;
        s.method = PSB_PCISPH;
        s.min_iters = s.max_iters = 3;
        s.particle_radius = 0.f;
        s.gravity[1] = -9.81f;
        if (psb_create(&s, &g_pci.ctx) != PSB_OK) {
            std::fprintf(stderr, "pci_SPH_update: psb_create failed; state not advanced\n");
            g_pci.ctx = nullptr;
            return;
        }
        g_pci.sc = s;
        g_pci.device = dev;
    }
    psb_ctx* c = g_pci.ctx;
    int rc = psb_upload_aos_f64(c, n, pos, vel, velInterAp, 1);
    if (rc == PSB_OK) rc = psb_step(c, 1);
    if (rc != PSB_OK) {
        std::fprintf(stderr, "pci_SPH_update: %s (%s); state not advanced\n", psb_status_string(rc), psb_last_error(c));
        return;
    }
    // the reference's final leap-frog leaves v- = v+ and x_old = x of the step's start
    cudaMemcpy(velInterAv, velInterAp, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice);
    cudaMemcpy(oldPos, pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice);
    psb_download_aos_f64(c, pos, nullptr, velInterAp, 1);
    if (g_pci.stage_n < n) {
        cudaFree(g_pci.stage);
        cudaMalloc((void**)&g_pci.stage, sizeof(float) * (size_t)n);
        g_pci.stage_n = n;
    }
    std::vector<float> h(n);
    psb_read_field(c, PSB_FIELD_DENSITY, h.data(), sizeof(float) * (size_t)n);
    cudaMemcpy(g_pci.stage, h.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
    k_copy_f32_to_f64<<<nblocks(n), kT>>>(g_pci.stage, density, n);
    psb_read_field(c, PSB_FIELD_PRESSURE, h.data(), sizeof(float) * (size_t)n);
    cudaMemcpy(g_pci.stage, h.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
    k_copy_f32_to_f64<<<nblocks(n), kT>>>(g_pci.stage, pressure, n);
    cudaDeviceSynchronize();
}

}  // extern "C"
