/*
 * refcuda_driver.cu -- runs the reference's own CUDA path on the GPU.
 *
 * BASELINE INFRASTRUCTURE ONLY (the bench's reference-cuda arm and a GPU
 * test). Built by oracle/Makefile (target refcuda) into
 * oracle/_ref/libpsbref_cuda.so from the reference sources where they lie,
 * compiled unchanged for sm_100a, plus this driver. The product never links
 * it.
 *
 * What is the reference's and what is ours:
 *  - the reference's: every kernel and pci_SPH_update, its PCISPH launcher
 *    (PciSphSystem.cu:8-68, with its per-call cudaMalloc/cudaFree and
 *    synchronisations), compiled from its files: UniformGridKernel.cu,
 *    SphKernel.cu, PciSphSystem_Kernel.cu, PciSphSystem.cu,
 *    BoxCollision_Kernel.cu, ForceExt_Constante.cu;
 *  - ours: device buffers in the reference's layouts (AoS double3,
 *    64-slot cells, 200-slot neighbour lists), computeGridSize (common.cu:
 *    102-107, 256-thread blocks), and the host call sequences of the files
 *    that do not compile without OpenGL or the XML loader:
 *    PCI_SPHSystem::update (PciSphSystem.cpp:163-204), SPHSystem::update
 *    (SphSystem.cpp:273-345 through SphSystem.cu:6-42), reinitCells,
 *    storeParticles, searchNeighbooring (UniformGrid.cu:64-99, with their
 *    launch shapes), collisionSystem_Box_CUDA (BoxCollision.cu:10-18),
 *    evaluate_ForceExt_Constante (ForceExt.cu:24-34).
 *
 * Guards the reference lacks. Its kernels write out of bounds for a particle
 * outside the grid (or not finite), for more than 64 particles in a cell and
 * for more than 200 neighbours (UniformGridKernel.cu:46-53, 82-85). Before
 * the grid is filled, one kernel of ours checks every position and counts
 * the cells' occupancy; after it is filled (in bounds by then), another
 * counts each particle's neighbours with the reference's test over the
 * reference's own slots. A step whose counts pass 64 per cell or 195 per
 * particle (5 below 200, so that no rounding of the test can reach 200)
 * returns a negative code before the reference's kernel that would write
 * past its arrays runs. The checks are outside the timed work.
 */
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <UniformGrid.cuh>
#include <UniformGridKernel.cuh>
#include <SphKernel.cuh>
#include <PciSphSystem.cuh>
#include <PciSphSystem_Kernel.cuh>
#include <BoxCollision_Kernel.cuh>
#include <ForceExt_Constante.cuh>

namespace {

constexpr int kMaxNbr = 200;        // listeVoisine stride, UniformGridKernel.cu:84
constexpr int kNbrGuard = 195;      // refused above this

struct Field {
    const char* name;
    int width;
};
const Field kFields[] = {
    {"pos_old", 3}, {"pos", 3}, {"vel_old", 3}, {"vel", 3}, {"vel_av", 3}, {"vel_ap", 3}, {"r_pos_old", 3},
    {"r_pos", 3}, {"r_vel_av", 3}, {"r_vel_ap", 3}, {"f_visc", 3}, {"f_surf", 3}, {"f_press", 3}, {"f_accum", 3},
    {"normals", 3}, {"mass", 1}, {"radius", 1}, {"rho0", 1}, {"k", 1}, {"mu", 1}, {"l", 1}, {"sigma", 1},
    {"density", 1}, {"density_err", 1}, {"pressure", 1},
};
constexpr int kNumFields = sizeof(kFields) / sizeof(kFields[0]);

__device__ int g_bad;          // a position outside the grid or not finite
__device__ int g_max_occ;      // largest cell occupancy
__device__ int g_max_nbr;      // largest neighbour count

// The cell storeParticles_Kernel computes (UniformGridKernel.cu:46-49),
// counted per cell; positions outside the grid are flagged instead.
__global__ void k_check_cells(const double3* pos, unsigned n, int* occ, float cell, float3 Min, int nx, int ny, int nz) {
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double3 x = pos[p];
    const double fi = floor((x.x - Min.x) / cell), fj = floor((x.y - Min.y) / cell), fk = floor((x.z - Min.z) / cell);
    if (!(fi >= 0 && fj >= 0 && fk >= 0 && fi < nx && fj < ny && fk < nz)) { g_bad = 1; return; }
    const long long c = (long long)fi + (long long)fj * nx + (long long)fk * nx * ny;
    atomicMax(&g_max_occ, atomicAdd(&occ[c], 1) + 1);
}

// Neighbour counts with searchNeighbooring_Kernel's test (UniformGridKernel.cu:
// 58-95) over the filled slots, without writing a list.
__global__ void k_check_neighbours(const double3* pos, const double* radius, const int* idx, const int* nb, int nx,
                                   int ny, int nz, float cell, float3 Min, unsigned n) {
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double3 x = pos[p];
    const int I = (int)floor((x.x - Min.x) / cell), J = (int)floor((x.y - Min.y) / cell),
              K = (int)floor((x.z - Min.z) / cell);
    int cnt = 0;
    for (int i = I - 1; i <= I + 1; ++i)
        for (int j = J - 1; j <= J + 1; ++j)
            for (int k = K - 1; k <= K + 1; ++k) {
                if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
                const long long c = i + (long long)j * nx + (long long)k * nx * ny;
                const int m = min(nb[c], MAXPARTICLES);
                for (int s = 0; s < m; ++s) {
                    const double3 y = pos[idx[c * MAXPARTICLES + s]];
                    const double dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
                    if (sqrt(dx * dx + dy * dy + dz * dz) <= radius[p]) ++cnt;
                }
            }
    atomicMax(&g_max_nbr, cnt);
}

}  // namespace

// The state of one reference scene on the device (handle of the rc_ API).
struct RefCudaSim {
    int n = 0;
    UniformGrid grid{};
    long long cells = 0;
    double* f[kNumFields] = {};
    int* nb_count = nullptr;
    int* nb_list = nullptr;
    int* occ = nullptr;
    cudaEvent_t ev[4] = {};
    std::string err;
};
typedef RefCudaSim Sim;

namespace {

double* field(Sim* s, const char* name, int* width) {
    for (int i = 0; i < kNumFields; ++i)
        if (!std::strcmp(name, kFields[i].name)) {
            if (width) *width = kFields[i].width;
            return s->f[i];
        }
    return nullptr;
}

template <typename T>
bool alloc(T** p, size_t count) {
    return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1)) == cudaSuccess;
}

unsigned blocks_for(unsigned n) { return (n + 255) / 256; }

// The grid part of PCI_SPHSystem::update and SPHSystem::update: reinitCells,
// storeParticles, searchNeighbooring (UniformGrid.cu:64-99) between the
// guards. Adds the reference's time to *ms.
int grid_and_lists(Sim* s, float* ms) {
    UniformGrid* g = &s->grid;
    const unsigned n = (unsigned)s->n;
    // guard 1: every position in the grid, at most MAXPARTICLES per cell
    const int zero = 0;
    cudaMemcpyToSymbol(g_bad, &zero, sizeof(int));
    cudaMemcpyToSymbol(g_max_occ, &zero, sizeof(int));
    cudaMemset(s->occ, 0, sizeof(int) * (size_t)s->cells);
    k_check_cells<<<blocks_for(n), 256>>>((const double3*)field(s, "pos", nullptr), n, s->occ, g->sizeCell, g->Min,
                                          g->nbCellsX, g->nbCellsY, g->nbCellsZ);
    int bad = 0, occ = 0;
    cudaMemcpyFromSymbol(&bad, g_bad, sizeof(int));
    cudaMemcpyFromSymbol(&occ, g_max_occ, sizeof(int));
    if (bad) { s->err = "a particle left the grid or is not finite"; return -2; }
    if (occ > MAXPARTICLES) { s->err = "a cell holds more than 64 particles"; return -3; }
    // reinitCells (UniformGrid.cu:64-76, its launch shape) and storeParticles (:80-87)
    int tx, bx, ty, by, tz, bz, t1, b1;
    computeGridSize(g->nbCellsX, bx, tx);
    computeGridSize(g->nbCellsY, by, ty);
    computeGridSize(g->nbCellsZ, bz, tz);
    computeGridSize((int)n, b1, t1);
    cudaEventRecord(s->ev[0]);
    reinitCells_Kernel<<<dim3(tx, ty, tz), dim3(bx, by, bz)>>>(g->nbParticles, g->nbCellsX, g->nbCellsY, g->nbCellsZ);
    storeParticles_Kernel<<<b1, t1>>>((double3*)field(s, "pos", nullptr), n, g->nbParticles, g->indexParticles,
                                      g->sizeCell, g->Min, g->nbCellsX, g->nbCellsY, g->nbCellsZ);
    cudaEventRecord(s->ev[1]);
    // guard 2: at most kNbrGuard neighbours per particle
    cudaMemcpyToSymbol(g_max_nbr, &zero, sizeof(int));
    k_check_neighbours<<<blocks_for(n), 256>>>((const double3*)field(s, "pos", nullptr), field(s, "radius", nullptr),
                                               g->indexParticles, g->nbParticles, g->nbCellsX, g->nbCellsY,
                                               g->nbCellsZ, g->sizeCell, g->Min, n);
    int nbr = 0;
    cudaMemcpyFromSymbol(&nbr, g_max_nbr, sizeof(int));
    float a = 0.f;
    cudaEventElapsedTime(&a, s->ev[0], s->ev[1]);
    *ms += a;
    if (nbr > kNbrGuard) { s->err = "a particle has more than 195 neighbours"; return -4; }
    partVoisine v{s->nb_count, s->nb_list};
    cudaEventRecord(s->ev[2]);
    searchNeighbooring_Kernel<<<b1, t1>>>((double3*)field(s, "pos", nullptr), field(s, "radius", nullptr),
                                          g->indexParticles, g->nbParticles, g->nbCellsX, g->nbCellsY, g->nbCellsZ,
                                          g->sizeCell, g->Min, 1.0, v, n);
    return 0;
}

// collide (BoxCollision.cu:10-18 through SPHSystem::collide, SphSystem.cpp:
// 323-328: pos, vel_av, vel_ap) and interpolateVelocities (SphSystem.cu:17-24)
void box_and_interpolate(Sim* s, float dt, float r, const float* bmin, const float* bmax) {
    int b, t;
    computeGridSize(s->n, b, t);
    collisionBox<<<b, t>>>(s->n, (double3*)field(s, "pos", nullptr), (double3*)field(s, "vel_av", nullptr),
                           (double3*)field(s, "vel_ap", nullptr), make_float3(bmin[0], bmin[1], bmin[2]),
                           make_float3(bmax[0], bmax[1], bmax[2]), 0.f, true, r, dt);
    interpolateSPH_velocities<<<b, t>>>((double3*)field(s, "vel_av", nullptr), (double3*)field(s, "vel_ap", nullptr),
                                        (double3*)field(s, "vel_old", nullptr), (double3*)field(s, "vel", nullptr),
                                        s->n);
}

}  // namespace

extern "C" {

// common.cu:102-107: 256-thread blocks
void computeGridSize(int n, int& numBlocks, int& numThreads) {
    const unsigned un = (unsigned)n;
    numThreads = (int)(un < 256u ? un : 256u);
    numBlocks = numThreads ? (int)((un + numThreads - 1) / numThreads) : 0;
}

Sim* rc_create(int n, const float* grid_min, float cell, const int* dims) {
    if (n <= 0 || !(cell > 0.f) || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return nullptr;
    Sim* s = new Sim();
    s->n = n;
    UniformGrid* g = &s->grid;
    g->Min = make_float3(grid_min[0], grid_min[1], grid_min[2]);
    g->sizeCell = cell;
    g->nbCellsX = dims[0];
    g->nbCellsY = dims[1];
    g->nbCellsZ = dims[2];
    g->Max = make_float3(grid_min[0] + dims[0] * cell, grid_min[1] + dims[1] * cell, grid_min[2] + dims[2] * cell);
    s->cells = (long long)dims[0] * dims[1] * dims[2];
    bool ok = alloc(&g->nbParticles, (size_t)s->cells) && alloc(&g->indexParticles, (size_t)s->cells * MAXPARTICLES) &&
              alloc(&s->occ, (size_t)s->cells) && alloc(&s->nb_count, (size_t)n) &&
              alloc(&s->nb_list, (size_t)n * kMaxNbr);
    for (int i = 0; ok && i < kNumFields; ++i) {
        ok = alloc(&s->f[i], (size_t)n * kFields[i].width);
        if (ok) ok = cudaMemset(s->f[i], 0, sizeof(double) * (size_t)n * kFields[i].width) == cudaSuccess;
    }
    if (ok) ok = cudaMemset(g->nbParticles, 0, sizeof(int) * (size_t)s->cells) == cudaSuccess;
    for (auto& e : s->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    if (!ok) {
        std::fprintf(stderr, "rc_create: device allocation failed\n");
        cudaGetLastError();
        return nullptr;
    }
    return s;
}

void rc_destroy(Sim* s) {
    if (!s) return;
    cudaDeviceSynchronize();
    for (auto p : s->f) cudaFree(p);
    cudaFree(s->grid.nbParticles);
    cudaFree(s->grid.indexParticles);
    cudaFree(s->occ);
    cudaFree(s->nb_count);
    cudaFree(s->nb_list);
    for (auto e : s->ev) if (e) cudaEventDestroy(e);
    delete s;
}

int rc_set(Sim* s, const char* name, const double* src) {
    int w = 0;
    double* d = field(s, name, &w);
    if (!d) return -1;
    return cudaMemcpy(d, src, sizeof(double) * (size_t)s->n * w, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -5;
}

int rc_get(Sim* s, const char* name, double* dst) {
    int w = 0;
    double* d = field(s, name, &w);
    if (!d) return -1;
    return cudaMemcpy(dst, d, sizeof(double) * (size_t)s->n * w, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -5;
}

int rc_neighbors(Sim* s, int* counts) {
    return cudaMemcpy(counts, s->nb_count, sizeof(int) * s->n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -5;
}

const char* rc_error(Sim* s) { return s ? s->err.c_str() : ""; }

// PCI_SPHSystem::update without emission (PciSphSystem.cpp:163-204): grid and
// lists, the reference's pci_SPH_update (its 3 corrections; threshold as the
// host driver of the reference kernels passes it), box, interpolation,
// restore copies. *ms: the reference's device time of the step.
int rc_pcisph_update(Sim* s, float dt, double threshold, float particle_radius, const float* bmin, const float* bmax,
                     float* ms) {
    float t = 0.f;
    const int rc = grid_and_lists(s, &t);
    if (rc) return rc;
    partVoisine v{s->nb_count, s->nb_list};
    auto F = [&](const char* k) { return field(s, k, nullptr); };
    pci_SPH_update(F("pos_old"), F("pos"), F("vel"), F("vel_av"), F("vel_ap"), F("r_pos_old"), F("r_pos"),
                   F("r_vel_av"), F("r_vel_ap"), F("mass"), F("radius"), F("density"), F("rho0"), F("density_err"),
                   F("pressure"), F("k"), F("mu"), F("l"), F("sigma"), threshold, v, F("normals"), F("f_visc"),
                   F("f_surf"), F("f_press"), F("f_accum"), dt, (uint)s->n);
    box_and_interpolate(s, dt, particle_radius, bmin, bmax);
    const size_t bytes = sizeof(double) * 3 * (size_t)s->n;
    cudaMemcpy(F("r_pos_old"), F("pos_old"), bytes, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F("r_pos"), F("pos"), bytes, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F("r_vel_av"), F("vel_av"), bytes, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F("r_vel_ap"), F("vel_ap"), bytes, cudaMemcpyDeviceToDevice);
    cudaEventRecord(s->ev[3]);
    cudaEventSynchronize(s->ev[3]);
    float a = 0.f;
    cudaEventElapsedTime(&a, s->ev[2], s->ev[3]);
    if (ms) *ms = t + a;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { s->err = cudaGetErrorString(e); return -5; }
    return 0;
}

// SPHSystem::update without emission (SphSystem.cpp:273-345): grid and lists,
// densityEvaluation and internalForces (SphSystem.cu:27-43), the constant
// force with the density as "mass" (ForceExt.cu:24-34), leap-frog
// (SphSystem.cu:6-14), box, interpolation.
int rc_wcsph_update(Sim* s, float dt, const float* gravity_dir, float gravity_amp, float particle_radius,
                    const float* bmin, const float* bmax, float* ms) {
    float t = 0.f;
    const int rc = grid_and_lists(s, &t);
    if (rc) return rc;
    partVoisine v{s->nb_count, s->nb_list};
    auto F = [&](const char* k) { return field(s, k, nullptr); };
    int b, th;
    computeGridSize(s->n, b, th);
    const unsigned n = (unsigned)s->n;
    densityEvaluation<<<b, th>>>((double3*)F("pos"), F("mass"), F("radius"), F("k"), F("rho0"), n, F("density"),
                                 F("pressure"), v);
    cudaDeviceSynchronize();
    internalForces<<<b, th>>>((double3*)F("pos"), (double3*)F("vel"), F("mass"), F("density"), F("pressure"),
                              F("radius"), F("mu"), F("l"), F("sigma"), (double3*)F("normals"), n,
                              (double3*)F("f_press"), (double3*)F("f_visc"), (double3*)F("f_surf"),
                              (double3*)F("f_accum"), v);
    cudaDeviceSynchronize();
    evaluate_force_constante<<<b, th>>>(n, (double3*)F("f_accum"), F("density"),
                                        make_float3(gravity_dir[0], gravity_dir[1], gravity_dir[2]), gravity_amp);
    cudaDeviceSynchronize();
    integrateSPH_LeapFrog<<<b, th>>>((double3*)F("vel_av"), (double3*)F("vel_ap"), (double3*)F("pos_old"),
                                     (double3*)F("pos"), (double3*)F("f_accum"), F("density"), dt, n);
    cudaDeviceSynchronize();
    box_and_interpolate(s, dt, particle_radius, bmin, bmax);
    cudaEventRecord(s->ev[3]);
    cudaEventSynchronize(s->ev[3]);
    float a = 0.f;
    cudaEventElapsedTime(&a, s->ev[2], s->ev[3]);
    if (ms) *ms = t + a;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { s->err = cudaGetErrorString(e); return -5; }
    return 0;
}

}  // extern "C"
