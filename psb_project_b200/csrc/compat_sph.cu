// compat_sph.cu -- the rest of the reference's extern "C" launchers that its
// system classes call (SPHSystem, PCI_SPHSystem, CudaSystem, SimpleSystem,
// SurfaceSPH), on the reference's own device layouts: WCSPH density and
// internal forces, the two external forces, the iso field and vertex normals
// over the reference's UniformGrid, the marching-cubes grid and polygonizer,
// and the common.cuh helpers.
//
// The kernels are FP64 restatements in the reference's expression order,
// compiled without multiply-add contraction (build.py), so that they agree
// with the reference's kernels to the last bits their math library calls
// (pow, powf, cos) leave. They read the caller's AoS double3 buffers, the
// 200-slot neighbour lists (partVoisine) and the 64-slot cells (UniformGrid)
// and never write past them: counts above the slots clamp and report once.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>

#include "psb.h"
#include "psb_compat.h"
#include "psb_internal.cuh"

namespace {

constexpr int kT = 256;
inline unsigned nblocks(long long n) { return (unsigned)((n + kT - 1) / kT); }
constexpr double kPi = 3.14159265358979323846;     // M_PI

__device__ int g_clamped;      // a count above the reference's slots was clamped

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 ld(const double* a, long long i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
__device__ __forceinline__ void st(double* a, long long i, D3 v) {
    a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z;
}
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
// double3.h: length = sqrt((x x + y y) + z z); a / s multiplies by 1 / s
__device__ __forceinline__ double len(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ D3 divv(D3 a, double s) { return mul(a, 1.0 / s); }

__device__ __forceinline__ int list_count(const partVoisine& v, long long i) {
    const int c = v.nbVoisines[i];
    if (c > PSB_COMPAT_MAX_NEIGHBOURS) { g_clamped = 1; return PSB_COMPAT_MAX_NEIGHBOURS; }
    return c;
}

// densityEvaluation (SphKernel.cu:9-27): rho_i = sum_j pow(h_j^2 - d^2, 3)
// 315 / (64 pi pow(h_j, 9)) m_j; p_i = k_i (rho_i - rho0_i)
__global__ void k_density(const double* pos, const double* mass, const double* radius, const double* k,
                          const double* rho0, int n, double* density, double* pressure, partVoisine v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const D3 xi = ld(pos, i);
    double rho = 0;
    const int cnt = list_count(v, i);
    for (int t = 0; t < cnt; ++t) {
        const long long j = v.listeVoisine[i * PSB_COMPAT_MAX_NEIGHBOURS + t];
        const double d = len(sub(xi, ld(pos, j)));
        const double a = 64 * kPi * pow(radius[j], 9);
        const double m_k = 315 / a;
        const double b = pow((radius[j] * radius[j]) - (d * d), 3);
        rho += b * m_k * mass[j];
    }
    density[i] = rho;
    pressure[i] = k[i] * (rho - rho0[i]);
}

// internalForces (SphKernel.cu:32-91): pressure, viscosity and surface
// tension force densities and the colour-field normal, summed over r > 0
__global__ void k_internal(const double* pos, const double* vel, const double* mass, const double* density,
                           const double* pressure, const double* radius, const double* visc, const double* l,
                           const double* sigma, double* normales, int n, double* f_p, double* f_v, double* f_s,
                           double* f_acc, partVoisine v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const D3 xi = ld(pos, i), vi = ld(vel, i);
    D3 fp{0, 0, 0}, fv{0, 0, 0}, nr{0, 0, 0};
    double fsurf = 0;
    const int cnt = list_count(v, i);
    for (int t = 0; t < cnt; ++t) {
        const long long j = v.listeVoisine[i * PSB_COMPAT_MAX_NEIGHBOURS + t];
        const D3 r = sub(xi, ld(pos, j));
        const double d = len(r);
        if (!(d > 0)) continue;
        const double h = radius[j];
        const D3 rn = divv(r, d);
        const double pV1 = pressure[i] / (density[i] * density[i]);
        const double pV2 = pressure[j] / (density[j] * density[j]);
        const double a = kPi * pow(h, 6);
        const D3 m_k = mul(rn, -45 * pow(h - d, 2) / a);
        fp = add(fp, mul(mul(m_k, pV1 + pV2), mass[j]));
        const double m_m = 45 * (h - d) / a;
        fv = add(fv, divv(mul(mul(mul(sub(ld(vel, j), vi), (visc[i] + visc[j]) / 2), mass[j]), m_m), density[j]));
        const double b = 32 * kPi * (double)powf((float)h, 9.f);
        const double m_d = -(945 / b) * ((h * h) - (d * d)) * ((3 * h * h) - (7 * d * d));
        fsurf += m_d * (mass[j] / density[j]);
        const double mk = -945 / b;
        nr = add(nr, mul(mul(mul(r, mass[j] / density[j]), pow((h * h) - (d * d), 2)), mk));
    }
    fp = mul(fp, -density[i]);
    const double lN = len(nr);
    D3 fs{0, 0, 0};
    if (lN >= l[i]) {
        fs = divv(mul(nr, fsurf * (-sigma[i])), lN);
        nr = {nr.x / lN, nr.y / lN, nr.z / lN};          // normalize: true divisions
    } else {
        nr = {0, 0, 0};
    }
    st(f_p, i, fp);
    st(f_v, i, fv);
    st(f_s, i, fs);
    st(normales, i, nr);
    st(f_acc, i, add(add(fv, fs), fp));
}

// evaluate_force_constante (ForceExt_Constante.cu:15-23): accum += (dir amp) m,
// the direction and amplitude in float as the launcher passes them
__global__ void k_force_constant(int n, double* accum, const double* mass, float3 dir, float amp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    accum[3 * i] += (double)(dir.x * amp) * mass[i];
    accum[3 * i + 1] += (double)(dir.y * amp) * mass[i];
    accum[3 * i + 2] += (double)(dir.z * amp) * mass[i];
}

// evaluate_force_trochoide (ForceExt_Trochoide.cu:14-24): a vertical force
// A cos(k (x cos theta + z sin theta) w t + phi) m on y
__global__ void k_force_trochoid(int n, const double* pos, double* accum, const double* mass, float A, float k,
                                 float theta, float w, float phi, float t) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const D3 x = ld(pos, i);
    const double val = A * cos(k * (x.x * (double)cosf(theta) + x.z * (double)sinf(theta)) * w * t + phi) * mass[i];
    accum[3 * i + 1] = accum[3 * i + 1] + val;
}

// The reference's UniformGrid cell of a point: floor((x - Min) / sizeCell) in FP64.
__device__ __forceinline__ void cell_ijk(D3 x, float3 Min, float cell, int& I, int& J, int& K) {
    I = (int)floor((x.x - Min.x) / cell);
    J = (int)floor((x.y - Min.y) / cell);
    K = (int)floor((x.z - Min.z) / cell);
}

__device__ __forceinline__ int cell_count(const int* counts, long long c) {
    const int m = counts[c];
    if (m > PSB_COMPAT_MAXPARTICLES) { g_clamped = 1; return PSB_COMPAT_MAXPARTICLES; }
    return m;
}

// evaluateIso_Kernel (UniformGridKernel.cu:98-138): at each node (double4,
// .w receives the value), sum over the particles of floor(1/scale) cell rings
// of (1/r^6) (r^2 - d^2)^3 for d <= r = h/scale, each term in float (powf)
__global__ void k_iso(double* node4, unsigned nx_mc, unsigned ny_mc, unsigned nz_mc, double scale, float3 Min,
                      float cell, int nx, int ny, int nz, const int* counts, const int* slots, const double* pos,
                      const double* radius, unsigned n) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)nx_mc * ny_mc * nz_mc) return;
    const D3 p1{node4[4 * c], node4[4 * c + 1], node4[4 * c + 2]};
    int I, J, K;
    cell_ijk(p1, Min, cell, I, J, K);
    const int ring = (int)floor(1 / scale);
    double iso = 0;
    for (int i = I - ring; i <= I + ring; ++i)
        for (int j = J - ring; j <= J + ring; ++j)
            for (int k = K - ring; k <= K + ring; ++k) {
                if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
                const long long cc = i + (long long)j * nx + (long long)k * nx * ny;
                const int m = cell_count(counts, cc);
                for (int s = 0; s < m; ++s) {
                    const unsigned q = (unsigned)slots[cc * PSB_COMPAT_MAXPARTICLES + s];
                    if (q >= n) continue;
                    const double r = radius[q] / scale;
                    const double d = len(sub(p1, ld(pos, q)));
                    if (d <= r) iso += (1 / powf((float)r, 6.f)) * powf((float)(r * r - d * d), 3.f);
                }
            }
    node4[4 * c + 3] = iso;
}

// computeNormales_Vertexs_Kernel (UniformGridKernel.cu:141-190): the colour-
// field gradient at each vertex over two cell rings, each listed term added
// six times as the reference's loop does, then -n/|n| (left at 0 when |n| is 0)
__global__ void k_vertex_normals(const double* posV, double* normales, float scale, unsigned nV, float3 Min, float cell,
                                 int nx, int ny, int nz, const int* counts, const int* slots, const double* pos,
                                 const double* radius, const double* mass, const double* density, unsigned n) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nV) return;
    const D3 p1 = ld(posV, v);
    int I, J, K;
    cell_ijk(p1, Min, cell, I, J, K);
    D3 nr{0, 0, 0};
    const int ring = 2;
    for (int i = I - ring; i <= I + ring; ++i)
        for (int j = J - ring; j <= J + ring; ++j)
            for (int k = K - ring; k <= K + ring; ++k) {
                if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
                const long long cc = i + (long long)j * nx + (long long)k * nx * ny;
                const int m = cell_count(counts, cc);
                for (int s = 0; s < m; ++s) {
                    const unsigned q = (unsigned)slots[cc * PSB_COMPAT_MAXPARTICLES + s];
                    if (q >= n) continue;
                    const double r = radius[q] / scale;
                    for (int rep = 0; rep < 6; ++rep) {
                        const D3 d12 = sub(p1, ld(pos, q));
                        const double d = len(d12);
                        if (d <= r) {
                            const double b = 32 * kPi * (double)powf((float)radius[q], 9.f);
                            const double mk = -945 / b;
                            nr = add(nr, mul(mul(mul(d12, mass[q] / density[q]),
                                                 pow((radius[q] * radius[q]) - (d * d), 2)), mk));
                        }
                    }
                }
            }
    const double lN = len(nr);
    st(normales, v, lN <= 0 ? nr : divv(D3{-nr.x, -nr.y, -nr.z}, lN));
}

// createGrid_MarchingCube_Kernel (MarchingCube_Kernel.cu:14-33): node centres
// C - L/2 + cell/2 + i cell (the last two terms in float), value 0, count 0
__global__ void k_mc_grid(double* node4, double cx, double cy, double cz, double l, double w, double d, float cell,
                          unsigned nx, unsigned ny, unsigned nz, int* counts) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)nx * ny * nz) return;
    const unsigned i = (unsigned)(c % nx), j = (unsigned)((c / nx) % ny), k = (unsigned)(c / ((long long)nx * ny));
    node4[4 * c] = cx - (l / 2) + (cell / 2) + i * cell;
    node4[4 * c + 1] = cy - (w / 2) + (cell / 2) + j * cell;
    node4[4 * c + 2] = cz - (d / 2) + (cell / 2) + k * cell;
    node4[4 * c + 3] = 0;
    counts[c] = 0;
}

void report(const char* where) {
    int f = 0;
    cudaMemcpyFromSymbol(&f, g_clamped, sizeof(int));
    if (f) {
        std::fprintf(stderr, "%s: a neighbour list above %d entries or a cell above %d particles was clamped\n", where,
                     PSB_COMPAT_MAX_NEIGHBOURS, PSB_COMPAT_MAXPARTICLES);
        const int z = 0;
        cudaMemcpyToSymbol(g_clamped, &z, sizeof(int));
    }
}

// The reference's ForceExt_Constante and ForceExt_Trochoide objects as the
// Itanium C++ ABI lays them out: the vtable pointer of their polymorphic
// base ForceExt (virtual draw()), then the members in declaration order.
struct ConstantForceLayout {          // ForceExt_Constante.h: Vector3 direction; float amplitude
    const void* vptr;
    double direction[3];              // Vector3: double e[3]
    float amplitude;
};
struct PeriodicForceLayout {          // ForceExt_Periodic.h: float A, lambda, k, theta, w, f, phi, time
    const void* vptr;
    float A, lambda, k, theta, w, f, phi, time;
};
static_assert(sizeof(ConstantForceLayout) == 40, "ForceExt_Constante layout");
static_assert(sizeof(PeriodicForceLayout) == 40, "ForceExt_Trochoide layout");

}  // namespace

extern "C" {

void evaluate_densities_forces(double* pos, double* vel, double* mass, double* radius, double* densities,
                               double* pressure, double* normales, double* restDensities, double* viscosities,
                               double* k, double* threshold, double* surfaceTension, int numBodies, double* fPressure,
                               double* fViscosity, double* fSurface, double* forcesAccum, partVoisine voisines) {
    if (numBodies <= 0) return;
    k_density<<<nblocks(numBodies), kT>>>(pos, mass, radius, k, restDensities, numBodies, densities, pressure, voisines);
    cudaDeviceSynchronize();
    k_internal<<<nblocks(numBodies), kT>>>(pos, vel, mass, densities, pressure, radius, viscosities, threshold,
                                           surfaceTension, normales, numBodies, fPressure, fViscosity, fSurface,
                                           forcesAccum, voisines);
    cudaDeviceSynchronize();
    report("evaluate_densities_forces");
}

void evaluate_ForceExt_Constante(unsigned int nbBodies, double* accumForceBuffer, double* mass,
                                 ForceExt_Constante* FC) {
    if (!nbBodies || !FC) return;
    const ConstantForceLayout* o = reinterpret_cast<const ConstantForceLayout*>(FC);
    const float3 dir = make_float3((float)o->direction[0], (float)o->direction[1], (float)o->direction[2]);
    k_force_constant<<<nblocks(nbBodies), kT>>>((int)nbBodies, accumForceBuffer, mass, dir, o->amplitude);
    cudaDeviceSynchronize();
}

void evaluate_ForceExt_Trochoide(unsigned int nbBodies, double* oldPos, double* accumForceBuffer, double* mass,
                                 ForceExt_Trochoide* T) {
    if (!nbBodies || !T) return;
    const PeriodicForceLayout* o = reinterpret_cast<const PeriodicForceLayout*>(T);
    k_force_trochoid<<<nblocks(nbBodies), kT>>>((int)nbBodies, oldPos, accumForceBuffer, mass, o->A, o->k, o->theta,
                                                o->w, o->phi, o->time);
    cudaDeviceSynchronize();
}

void evaluateIso_CUDA(double* posMC, unsigned int nbCellsX_MC, unsigned int nbCellsY_MC, unsigned int nbCellsZ_MC,
                      double scale, UniformGrid* grid, double* pos, double* radius, unsigned int nbBodies) {
    const long long nn = (long long)nbCellsX_MC * nbCellsY_MC * nbCellsZ_MC;
    if (nn <= 0 || !(scale > 0) || scale < 1.0 / 16) {
        if (nn > 0) std::fprintf(stderr, "evaluateIso_CUDA: scale %g outside [1/16, inf): not evaluated\n", scale);
        return;
    }
    k_iso<<<nblocks(nn), kT>>>(posMC, nbCellsX_MC, nbCellsY_MC, nbCellsZ_MC, scale, grid->Min, grid->sizeCell,
                               grid->nbCellsX, grid->nbCellsY, grid->nbCellsZ, grid->nbParticles, grid->indexParticles,
                               pos, radius, nbBodies);
    cudaDeviceSynchronize();
    report("evaluateIso_CUDA");
}

void computeNormales_Vertex_CUDA(double* posV, double* normales, float scale, unsigned int nbV, UniformGrid* grid,
                                 double* pos, double* radius, double* mass, double* densities, unsigned int nbBodies) {
    if (!nbV) return;
    k_vertex_normals<<<nblocks(nbV), kT>>>(posV, normales, scale, nbV, grid->Min, grid->sizeCell, grid->nbCellsX,
                                           grid->nbCellsY, grid->nbCellsZ, grid->nbParticles, grid->indexParticles, pos,
                                           radius, mass, densities, nbBodies);
    cudaDeviceSynchronize();
    report("computeNormales_Vertex_CUDA");
}

void createGrid_MarchingCube_CUDA(psb_vec3_arg C, double l, double w, double d, float sizeCell, unsigned int nbPosX,
                                  unsigned int nbPosY, unsigned int nbPosZ, double* grid, int* m_nbIndex) {
    const long long nn = (long long)nbPosX * nbPosY * nbPosZ;
    if (nn <= 0) return;
    k_mc_grid<<<nblocks(nn), kT>>>(grid, C.e[0], C.e[1], C.e[2], l, w, d, sizeCell, nbPosX, nbPosY, nbPosZ, m_nbIndex);
    cudaDeviceSynchronize();
}

void polygonize_MarchingCube_CUDA(double* grid, unsigned int nbPosX, unsigned int nbPosY, unsigned int nbPosZ,
                                  double isoLevel, int* m_nbIndex, double* m_vertex, double* m_normales, int* m_index) {
    (void)m_normales;    // the reference's kernel does not write it either
    if (nbPosX < 2 || nbPosY < 2 || nbPosZ < 2) return;
    psb::mc_upload_table(0);
    psb::launch_mc_polygonize_slots(0, grid, (int)nbPosX, (int)nbPosY, (int)nbPosZ, isoLevel, m_nbIndex, m_vertex,
                                    m_index, PSB_COMPAT_MC_SLOTS);
    cudaDeviceSynchronize();
}

void displayGrid(UniformGrid* grid) {
    (void)grid;    // drawing the grid is the GUI's (OpenGL); there is nothing to draw headless
}

// ---- common.cuh ------------------------------------------------------------------
int getCudaEnabledDeviceCount(void) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e == cudaErrorNoDevice) return 0;
    if (e == cudaErrorInsufficientDriver) return -1;
    return e == cudaSuccess ? count : 0;
}
int getcudaEnabledDeviceCount(void) { return getCudaEnabledDeviceCount(); }

bool cudaInit(int argc, char** argv) {
    (void)argc; (void)argv;
    int dev = 0;
    if (getCudaEnabledDeviceCount() <= 0 || cudaGetDevice(&dev) != cudaSuccess) {
        std::fprintf(stderr, "cudaInit: no CUDA device\n");
        return false;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
        std::printf("GPU Device %d: \"%s\" with compute capability %d.%d\n\n", dev, prop.name, prop.major, prop.minor);
    return true;
}

void cudaGLInit(int argc, char** argv) { (void)cudaInit(argc, argv); }

void allocateArray(void** devPtr, size_t size) {
    if (cudaMalloc(devPtr, size) != cudaSuccess) {
        cudaGetLastError();
        *devPtr = nullptr;
        std::fprintf(stderr, "allocateArray: cudaMalloc of %zu bytes failed\n", size);
    }
}

void freeArray(void* devPtr) { cudaFree(devPtr); }

void threadSync(void) { cudaDeviceSynchronize(); }

void copyArrayToDevice(void* device, const void* host, int offset, int size) {
    cudaMemcpy((char*)device + offset, host, (size_t)size, cudaMemcpyHostToDevice);
}

void copyArrayDeviceToDevice(void* device, const void* host, int offset, int size) {
    cudaMemcpy((char*)device + offset, host, (size_t)size, cudaMemcpyDeviceToDevice);
}

void copyArrayFromDevice(void* host, const void* device, struct cudaGraphicsResource** cuda_vbo_resource, int size) {
    (void)cuda_vbo_resource;     // the reference does not map it either (common.cu:86-91)
    cudaMemcpy(host, device, (size_t)size, cudaMemcpyDeviceToHost);
}

int iDivUp(int a, int b) {
    const unsigned ua = (unsigned)a, ub = (unsigned)b;     // common.cu computes in unsigned
    return ub == 0 ? 0 : (int)((ua % ub != 0) ? (ua / ub + 1) : (ua / ub));
}

void computeGridSize(int n, int& numBlocks, int& numThreads) {
    const unsigned un = (unsigned)n;
    numThreads = (int)(un < 256u ? un : 256u);
    numBlocks = iDivUp(n, numThreads);      // 0 blocks for n = 0 (the reference divides by zero there)
}

}  // extern "C"
