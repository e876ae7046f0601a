/*
 * ref_driver.cpp -- runs the reference's own device kernels on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Built by oracle/Makefile into
 * oracle/_ref/libpsbref.so from the reference sources, where they lie, plus
 * this driver and ref_shim.h. It is the pinned checker for the reference-
 * compatible physics profile and the "reference" CPU baseline; the product
 * never links it.
 *
 * What is the reference's and what is ours:
 *  - every floating-point expression on the path is the reference's kernel
 *    body, compiled unchanged: storeParticles_Kernel/searchNeighbooring_Kernel
 *    (src/Utils/Neighborhood/UniformGrid/UniformGridKernel.cu:43-95),
 *    densityEvaluation, internalForces, integrateSPH_LeapFrog(_Forces) and
 *    interpolateSPH_velocities (SphKernel.cu:9-135),
 *    the compute_..._PCI kernels and restore_Pos_Vel_PCI (PciSphSystem_Kernel.cu:36-201),
 *    collisionBox (BoxCollision_Kernel.cu:7-34), evaluate_force_constante
 *    (ForceExt_Constante.cu:15-23), collideParticles (CudaParticle_Kernel.cu:42-55),
 *    integrateEuler (ParticleKernel.cu:12-20);
 *  - this file restates, in our own code, the host launchers' call sequences
 *    (PciSphSystem.cu:8-68, PciSphSystem.cpp:163-204, SphSystem.cpp:273-345,
 *    SphSystem.cu:6-42, UniformGrid.cu:64-99, BoxCollision.cu:10-18,
 *    CudaSystem.cpp:207-250, ForceExt.cu:24-34) and the launch sizing of
 *    computeGridSize (common.cu:102-107: 256-thread blocks).
 *
 * Differences from running the reference on a GPU, all below the tolerances
 * the tests use: no FMA contraction on the host (-ffp-contract=off), and
 * glibc pow/powf/sqrt in place of CUDA's. Bucket slot order inside a cell is
 * deterministic here (storeParticles runs on one host thread, so slots fill
 * in increasing particle index); on a GPU it follows atomicAdd order.
 *
 * Safety checks the reference lacks (it writes out of bounds instead): a
 * particle outside the grid, more than MAXPARTICLES (64) in a cell, or more
 * than 200 neighbours makes the call return a negative code.
 */
#include "ref_shim.h"
#include <UniformGrid.cuh>
#include <UniformGridKernel.cuh>
#include <SphKernel.cuh>
#include <PciSphSystem_Kernel.cuh>
#include <CudaParticle_Kernel.cuh>
#include <MarchingCube.cuh>
#include <vector>
#include <string>
#include <cstdlib>

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

/* Kernels compiled from .cu files without an extern "C" header of their own. */
void collisionBox(int nbBodies, double3* newPos, double3* oldVel, double3* newVel, float3 Min, float3 Max,
                  float elast, bool container, float radiusParticles, float dt);
void evaluate_force_constante(uint nbBodies, double3* accumForceBuff, double* mass, float3 direction, float amplitude);
void evaluate_force_trochoide(uint nbBodies, double3* position, double3* accumForceBuff, double* mass, float A, float k,
                              float theta, float w, float phi, float t);
void integrateEuler(uint nbBodies, double3* newPos, double3* newVel, double3* forces, double* mass, float dt);
/* The collision objects' kernels (src/Kernel/Collision/*), C++ linkage
 * where their headers have no extern "C". */
void collisionPlan(uint nbBodies, double3* newPos, double3* newVel, double3* oldPos, double3* oldVel, float3 A,
                   float3 B, float3 C, float3 D, float3 N, float elast, float dt);
void collisionSphere(uint nbBodies, double3* newPos, double3* newVel, double3* oldPos, double3* oldVel, float3 origin,
                     float radius, float elast, bool container, float dt);
void collisionCylinder(int nbBodies, double3* newPos, double3* newVel, float radiusParticle, float dt, float elast,
                       bool container, float3 center, float baseRadius, float length, float3 direction);
extern "C" void collisionTriangle(uint nbBodies, uint nbFaces, double3* newPos, double3* newVel, double3* oldPos,
                                  double3* oldVel, float* AF, float* BF, float* CF, float* NF, float elast,
                                  float radiusParticle, float dt);
extern "C" void collisionSystem_Linear_HeightFieldCollision_Kernel(double3* newPos, double3* newVel,
                                                                   double radiusParticle, float dt, uint nbBodiesP,
                                                                   double a, double b, float3 min_, float3 max_,
                                                                   float elast);
extern "C" void collisionSystem_Gaussian_HeightFieldCollision_Kernel(double3* newPos, double3* newVel,
                                                                     double radiusParticle, float dt, uint nbBodiesP,
                                                                     double A, double x0, double z0, double p1,
                                                                     double p2, float3 min_, float3 max_, float elast);
extern "C" void collisionSystem_Periodic_HeightFieldCollision_Kernel(double3* newPos, double3* newVel,
                                                                     double radiusParticle, float dt, uint nbBodiesP,
                                                                     uint nbFunc, double* A, double* k, double* theta,
                                                                     double* phi, float3 min_, float3 max_,
                                                                     float elast);
/* MarchingCube_Kernel.cu:36 (its header also defines the case tables, which
 * that file's object already holds) */
extern "C" void polygonize_MarchingCube_Kernel(double4* grid, uint nbCellsX, uint nbCellsY, uint nbCellsZ,
                                               double isoLevel, int* nbIndex, double3* vertexs, double3* normales,
                                               int* indexs);
extern "C" void createGrid_MarchingCube_Kernel(double4* grid, double3 center, double l, double w, double d,
                                               float sizeCell, uint nbPosX, uint nbPosY, uint nbPosZ, int* m_nbIndex);

namespace {

const int kMaxNbr = 200;   /* listeVoisine stride, UniformGridKernel.cu:84 */

/* Emulates kernel<<<ceil(n/256), min(256,n)>>> (computeGridSize, common.cu:102-107).
 * Blocks are spread over host threads; the reference kernels have no
 * intra-block communication, so any schedule gives the same results. */
template <typename F>
void launch1d(unsigned n, bool parallel, F body) {
    if (n == 0) return;
    const unsigned threads = n < 256u ? n : 256u;
    const long blocks = (long)((n + threads - 1) / threads);
#pragma omp parallel for schedule(static) if (parallel)
    for (long b = 0; b < blocks; ++b) {
        blockIdx = make_uint3((unsigned)b, 0, 0);
        blockDim = dim3(threads, 1, 1);
        gridDim = dim3((unsigned)blocks, 1, 1);
        for (unsigned t = 0; t < threads; ++t) {
            threadIdx = make_uint3(t, 0, 0);
            body();
        }
    }
}

/* One host thread per cell (grid of cells, 1-thread blocks), as the
 * reference's "3D-swapped" launches end up (UniformGrid.cu:64-77). */
template <typename F>
void launch_cells(int nx, int ny, int nz, F body) {
#pragma omp parallel for schedule(static)
    for (long z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                blockIdx = make_uint3(x, y, (unsigned)z);
                blockDim = dim3(1, 1, 1);
                threadIdx = make_uint3(0, 0, 0);
                body();
            }
}

}  // namespace

struct ref_sim {
    int n = 0;
    UniformGrid grid{};
    std::vector<int> cell_idx, cell_nb;
    std::vector<int> nb_count, nb_list;
    /* AoS double3 particle arrays (stride 3), as the reference's m_d* buffers. */
    std::vector<double> pos_old, pos, vel_old, vel, vel_av, vel_ap;
    std::vector<double> r_pos_old, r_pos, r_vel_av, r_vel_ap;      /* restore buffers */
    std::vector<double> f_visc, f_surf, f_press, f_accum, normals;
    /* per-particle scalars */
    std::vector<double> mass, radius, rho0, k, mu, l, sigma, density, density_err, pressure, threshold;
    /* DEM coefficients */
    std::vector<double> spring, damping, shear, attraction;
};

static std::vector<double>* field(ref_sim* s, const char* name, int* width) {
    struct E { const char* n; std::vector<double> ref_sim::*p; int w; };
    static const E table[] = {
        {"pos_old", &ref_sim::pos_old, 3}, {"pos", &ref_sim::pos, 3}, {"vel_old", &ref_sim::vel_old, 3},
        {"vel", &ref_sim::vel, 3}, {"vel_av", &ref_sim::vel_av, 3}, {"vel_ap", &ref_sim::vel_ap, 3},
        {"r_pos_old", &ref_sim::r_pos_old, 3}, {"r_pos", &ref_sim::r_pos, 3},
        {"r_vel_av", &ref_sim::r_vel_av, 3}, {"r_vel_ap", &ref_sim::r_vel_ap, 3},
        {"f_visc", &ref_sim::f_visc, 3}, {"f_surf", &ref_sim::f_surf, 3}, {"f_press", &ref_sim::f_press, 3},
        {"f_accum", &ref_sim::f_accum, 3}, {"normals", &ref_sim::normals, 3},
        {"mass", &ref_sim::mass, 1}, {"radius", &ref_sim::radius, 1}, {"rho0", &ref_sim::rho0, 1},
        {"k", &ref_sim::k, 1}, {"mu", &ref_sim::mu, 1}, {"l", &ref_sim::l, 1}, {"sigma", &ref_sim::sigma, 1},
        {"density", &ref_sim::density, 1}, {"density_err", &ref_sim::density_err, 1},
        {"pressure", &ref_sim::pressure, 1}, {"threshold", &ref_sim::threshold, 1},
        {"spring", &ref_sim::spring, 1}, {"damping", &ref_sim::damping, 1}, {"shear", &ref_sim::shear, 1},
        {"attraction", &ref_sim::attraction, 1},
    };
    for (const E& e : table)
        if (std::string(name) == e.n) { *width = e.w; return &(s->*(e.p)); }
    return nullptr;
}

extern "C" {

/* Grid as createGrid sets it (UniformGrid.cu:17-49), given directly by its
 * float Min corner, float cell size and cell counts. */
ref_sim* ref_create(int n, const float* grid_min, float cell, const int* dims) {
    if (n <= 0 || cell <= 0.f || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return nullptr;
    ref_sim* s = new ref_sim();
    s->n = n;
    s->grid.Min = make_float3(grid_min[0], grid_min[1], grid_min[2]);
    s->grid.sizeCell = cell;
    s->grid.nbCellsX = dims[0];
    s->grid.nbCellsY = dims[1];
    s->grid.nbCellsZ = dims[2];
    s->grid.Max = make_float3(grid_min[0] + dims[0] * cell, grid_min[1] + dims[1] * cell, grid_min[2] + dims[2] * cell);
    const size_t cells = (size_t)dims[0] * dims[1] * dims[2];
    s->cell_nb.assign(cells, 0);
    s->cell_idx.assign(cells * MAXPARTICLES, 0);
    s->grid.nbParticles = s->cell_nb.data();
    s->grid.indexParticles = s->cell_idx.data();
    s->nb_count.assign(n, 0);
    s->nb_list.assign((size_t)n * kMaxNbr + 27 * MAXPARTICLES, 0);
    for (auto* v : {&s->pos_old, &s->pos, &s->vel_old, &s->vel, &s->vel_av, &s->vel_ap, &s->r_pos_old, &s->r_pos,
                    &s->r_vel_av, &s->r_vel_ap, &s->f_visc, &s->f_surf, &s->f_press, &s->f_accum, &s->normals})
        v->assign((size_t)n * 3, 0.0);
    for (auto* v : {&s->mass, &s->radius, &s->rho0, &s->k, &s->mu, &s->l, &s->sigma, &s->density, &s->density_err,
                    &s->pressure, &s->threshold, &s->spring, &s->damping, &s->shear, &s->attraction})
        v->assign((size_t)n, 0.0);
    return s;
}

void ref_destroy(ref_sim* s) { delete s; }

int ref_set(ref_sim* s, const char* name, const double* src) {
    int w = 0;
    std::vector<double>* v = field(s, name, &w);
    if (!v) return -1;
    std::memcpy(v->data(), src, sizeof(double) * v->size());
    return 0;
}

int ref_get(ref_sim* s, const char* name, double* dst) {
    int w = 0;
    std::vector<double>* v = field(s, name, &w);
    if (!v) return -1;
    std::memcpy(dst, v->data(), sizeof(double) * v->size());
    return 0;
}

/* reinitCells + storeParticles + searchNeighbooring (UniformGrid.cu:64-99),
 * called as SPHSystem/PCI_SPHSystem::update do with scale 1
 * (PciSphSystem.cpp:168-170). Returns 0, or -2 (particle outside the grid),
 * -3 (cell over MAXPARTICLES), -4 (more than 200 neighbours). */
int ref_search(ref_sim* s) {
    UniformGrid* g = &s->grid;
    /* Range check first: storeParticles_Kernel has none (UniformGridKernel.cu:46-53). */
    for (int i = 0; i < s->n; ++i) {
        const double* p = &s->pos[3 * (size_t)i];
        int c[3];
        c[0] = (int)floor((p[0] - g->Min.x) / g->sizeCell);
        c[1] = (int)floor((p[1] - g->Min.y) / g->sizeCell);
        c[2] = (int)floor((p[2] - g->Min.z) / g->sizeCell);
        if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= g->nbCellsX || c[1] >= g->nbCellsY || c[2] >= g->nbCellsZ)
            return -2;
    }
    launch_cells(g->nbCellsX, g->nbCellsY, g->nbCellsZ,
                 [&] { reinitCells_Kernel(g->nbParticles, g->nbCellsX, g->nbCellsY, g->nbCellsZ); });
    /* Counts are checked before the slots are written. */
    {
        std::vector<int> cnt(s->cell_nb.size(), 0);
        for (int i = 0; i < s->n; ++i) {
            const double* p = &s->pos[3 * (size_t)i];
            int a = (int)floor((p[0] - g->Min.x) / g->sizeCell);
            int b = (int)floor((p[1] - g->Min.y) / g->sizeCell);
            int c = (int)floor((p[2] - g->Min.z) / g->sizeCell);
            if (++cnt[(size_t)a + (size_t)b * g->nbCellsX + (size_t)c * g->nbCellsX * g->nbCellsY] > MAXPARTICLES)
                return -3;
        }
    }
    launch1d(s->n, false, [&] {
        storeParticles_Kernel((double3*)s->pos.data(), s->n, g->nbParticles, g->indexParticles, g->sizeCell, g->Min,
                              g->nbCellsX, g->nbCellsY, g->nbCellsZ);
    });
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    /* The kernel appends without a bound (UniformGridKernel.cu:82-85). The
     * list is padded by the most one particle can append (27 cells x 64
     * slots), so an overflow stays inside the allocation; the count check
     * below then rejects the call. */
    launch1d(s->n, true, [&] {
        searchNeighbooring_Kernel((double3*)s->pos.data(), s->radius.data(), g->indexParticles, g->nbParticles,
                                  g->nbCellsX, g->nbCellsY, g->nbCellsZ, g->sizeCell, g->Min, 1.0, v, s->n);
    });
    for (int i = 0; i < s->n; ++i)
        if (s->nb_count[i] > kMaxNbr) return -4;
    return 0;
}

int ref_neighbors(ref_sim* s, int* counts, int* list) {
    std::memcpy(counts, s->nb_count.data(), sizeof(int) * s->n);
    if (list) std::memcpy(list, s->nb_list.data(), sizeof(int) * (size_t)s->n * kMaxNbr);
    return 0;
}

int ref_cell_counts(ref_sim* s, int* counts) {
    std::memcpy(counts, s->cell_nb.data(), sizeof(int) * s->cell_nb.size());
    return 0;
}

/* compute_Density_PCI at the current positions over the current lists. */
int ref_density_pci(ref_sim* s) {
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    launch1d(s->n, true, [&] {
        compute_Density_PCI(s->n, (double3*)s->pos.data(), s->mass.data(), s->radius.data(), s->density.data(),
                            s->rho0.data(), s->density_err.data(), v);
    });
    return 0;
}

/* pci_SPH_update (PciSphSystem.cu:8-68), kernel for kernel; `iters` is the
 * reference's fixed 3 unless a test asks otherwise. */
static void pci_sph_update(ref_sim* s, float dt, int iters) {
    const uint n = s->n;
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    double3* pos = (double3*)s->pos.data();
    launch1d(n, true, [&] {
        compute_Density_PCI(n, pos, s->mass.data(), s->radius.data(), s->density.data(), s->rho0.data(),
                            s->density_err.data(), v);
    });
    launch1d(n, true, [&] {
        compute_Viscosity_SurfaceTension_Force_PCI(n, pos, (double3*)s->vel.data(), s->mass.data(), s->density.data(),
                                                   s->pressure.data(), s->radius.data(), s->mu.data(), s->threshold.data(),
                                                   s->sigma.data(), (double3*)s->normals.data(), (double3*)s->f_press.data(),
                                                   (double3*)s->f_visc.data(), (double3*)s->f_surf.data(),
                                                   (double3*)s->f_accum.data(), v);
    });
    for (int it = 0; it < iters; ++it) {
        launch1d(n, true, [&] {
            integrateSPH_LeapFrog_Forces((double3*)s->vel_av.data(), (double3*)s->vel_ap.data(), (double3*)s->pos_old.data(),
                                         pos, (double3*)s->f_visc.data(), (double3*)s->f_surf.data(),
                                         (double3*)s->f_press.data(), (double3*)s->f_accum.data(), s->density.data(), dt, n);
        });
        launch1d(n, true, [&] {
            compute_Density_PCI(n, pos, s->mass.data(), s->radius.data(), s->density.data(), s->rho0.data(),
                                s->density_err.data(), v);
        });
        launch1d(n, true, [&] {
            compute_Pressure_PCI(n, pos, s->mass.data(), s->radius.data(), s->k.data(), 10.0, s->density.data(),
                                 s->rho0.data(), s->density_err.data(), s->pressure.data(), v, dt);
        });
        launch1d(n, true, [&] {
            compute_Pressure_Force_PCI(n, pos, s->mass.data(), s->density.data(), s->rho0.data(), s->density_err.data(),
                                       s->pressure.data(), s->radius.data(), (double3*)s->f_press.data(), 10.0, v);
        });
        launch1d(n, true, [&] {
            restore_Pos_Vel_PCI((double3*)s->r_vel_av.data(), (double3*)s->r_vel_ap.data(), (double3*)s->r_pos_old.data(),
                                (double3*)s->r_pos.data(), (double3*)s->vel_av.data(), (double3*)s->vel_ap.data(),
                                (double3*)s->pos_old.data(), pos, n);
        });
    }
    launch1d(n, true, [&] {
        integrateSPH_LeapFrog_Forces((double3*)s->vel_av.data(), (double3*)s->vel_ap.data(), (double3*)s->pos_old.data(),
                                     pos, (double3*)s->f_visc.data(), (double3*)s->f_surf.data(), (double3*)s->f_press.data(),
                                     (double3*)s->f_accum.data(), s->density.data(), dt, n);
    });
}

static void collide_box(ref_sim* s, float particle_radius, float dt, const float* box_min, const float* box_max) {
    /* BoxCollision::collide -> collisionSystem_Box_CUDA (BoxCollision.cpp:34-37,
     * BoxCollision.cu:10-18), acting on (pos, vel_av, vel_ap) as
     * SPHSystem::collide passes them (SphSystem.cpp:323-328). */
    launch1d(s->n, true, [&] {
        collisionBox(s->n, (double3*)s->pos.data(), (double3*)s->vel_av.data(), (double3*)s->vel_ap.data(),
                     make_float3(box_min[0], box_min[1], box_min[2]), make_float3(box_max[0], box_max[1], box_max[2]),
                     0.f, true, particle_radius, dt);
    });
}

static void interpolate(ref_sim* s) {
    launch1d(s->n, true, [&] {
        interpolateSPH_velocities((double3*)s->vel_av.data(), (double3*)s->vel_ap.data(), (double3*)s->vel_old.data(),
                                  (double3*)s->vel.data(), s->n);
    });
}

/* PCI_SPHSystem::update without emission (PciSphSystem.cpp:163-204).
 * `collide` = 0 skips the box (a scene without collision objects). */
int ref_pcisph_update(ref_sim* s, float dt, int iters, int collide, float particle_radius,
                      const float* box_min, const float* box_max) {
    int rc = ref_search(s);
    if (rc) return rc;
    pci_sph_update(s, dt, iters);
    if (collide) collide_box(s, particle_radius, dt, box_min, box_max);
    interpolate(s);
    s->r_pos_old = s->pos_old;
    s->r_pos = s->pos;
    s->r_vel_av = s->vel_av;
    s->r_vel_ap = s->vel_ap;
    return 0;
}

/* SPHSystem::update without emission (SphSystem.cpp:273-297): density and
 * internal forces (SphSystem.cu:27-42), the constant external force with the
 * density passed as "mass" (SphSystem.cpp:307-320, ForceExt.cu:24-34),
 * leap-frog (SphSystem.cu:6-14), box, velocity interpolation. */
int ref_wcsph_update(ref_sim* s, float dt, const float* gravity_dir, float gravity_amp, int collide,
                     float particle_radius, const float* box_min, const float* box_max) {
    int rc = ref_search(s);
    if (rc) return rc;
    const uint n = s->n;
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    double3* pos = (double3*)s->pos.data();
    launch1d(n, true, [&] {
        densityEvaluation(pos, s->mass.data(), s->radius.data(), s->k.data(), s->rho0.data(), n, s->density.data(),
                          s->pressure.data(), v);
    });
    launch1d(n, true, [&] {
        internalForces(pos, (double3*)s->vel.data(), s->mass.data(), s->density.data(), s->pressure.data(),
                       s->radius.data(), s->mu.data(), s->threshold.data(), s->sigma.data(), (double3*)s->normals.data(), n,
                       (double3*)s->f_press.data(), (double3*)s->f_visc.data(), (double3*)s->f_surf.data(),
                       (double3*)s->f_accum.data(), v);
    });
    const float3 dir = make_float3(gravity_dir[0], gravity_dir[1], gravity_dir[2]);
    launch1d(n, true, [&] { evaluate_force_constante(n, (double3*)s->f_accum.data(), s->density.data(), dir, gravity_amp); });
    launch1d(n, true, [&] {
        integrateSPH_LeapFrog((double3*)s->vel_av.data(), (double3*)s->vel_ap.data(), (double3*)s->pos_old.data(), pos,
                              (double3*)s->f_accum.data(), s->density.data(), dt, n);
    });
    if (collide) collide_box(s, particle_radius, dt, box_min, box_max);
    interpolate(s);
    return 0;
}

/* CudaSystem::update without emission (CudaSystem.cpp:207-250): forces
 * zeroed, gravity m*g, pair forces on (pos_old, vel_old), explicit Euler on
 * (pos, vel), box. Tests call it with pos_old == pos and vel_old == vel. */
int ref_dem_update(ref_sim* s, float dt, const float* gravity_dir, float gravity_amp, int collide,
                   float particle_radius, const float* box_min, const float* box_max) {
    int rc = ref_search(s);
    if (rc) return rc;
    const uint n = s->n;
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    std::fill(s->f_accum.begin(), s->f_accum.end(), 0.0);
    const float3 dir = make_float3(gravity_dir[0], gravity_dir[1], gravity_dir[2]);
    launch1d(n, true, [&] { evaluate_force_constante(n, (double3*)s->f_accum.data(), s->mass.data(), dir, gravity_amp); });
    launch1d(n, true, [&] {
        collideParticles(n, (double3*)s->pos_old.data(), (double3*)s->vel_old.data(), (double3*)s->f_accum.data(),
                         s->radius.data(), s->spring.data(), s->damping.data(), s->shear.data(), s->attraction.data(), v);
    });
    launch1d(n, true, [&] {
        integrateEuler(n, (double3*)s->pos.data(), (double3*)s->vel.data(), (double3*)s->f_accum.data(), s->mass.data(), dt);
    });
    if (collide) {
        launch1d(n, true, [&] {
            collisionBox(n, (double3*)s->pos.data(), (double3*)s->vel_old.data(), (double3*)s->vel.data(),
                         make_float3(box_min[0], box_min[1], box_min[2]), make_float3(box_max[0], box_max[1], box_max[2]),
                         0.f, true, particle_radius, dt);
        });
    }
    return 0;
}

/* evaluate_densities_forces (SphSystem.cu:27-43): densityEvaluation then
 * internalForces over the lists of the current positions (grid rebuilt). */
int ref_densities_forces(ref_sim* s) {
    int rc = ref_search(s);
    if (rc) return rc;
    const uint n = s->n;
    partVoisine v{s->nb_count.data(), s->nb_list.data()};
    double3* pos = (double3*)s->pos.data();
    launch1d(n, true, [&] {
        densityEvaluation(pos, s->mass.data(), s->radius.data(), s->k.data(), s->rho0.data(), n, s->density.data(),
                          s->pressure.data(), v);
    });
    launch1d(n, true, [&] {
        internalForces(pos, (double3*)s->vel.data(), s->mass.data(), s->density.data(), s->pressure.data(),
                       s->radius.data(), s->mu.data(), s->threshold.data(), s->sigma.data(), (double3*)s->normals.data(), n,
                       (double3*)s->f_press.data(), (double3*)s->f_visc.data(), (double3*)s->f_surf.data(),
                       (double3*)s->f_accum.data(), v);
    });
    return 0;
}

/* computeNormales_Vertex_CUDA -> computeNormales_Vertexs_Kernel
 * (UniformGridKernel.cu:141-190) at nV vertices (xyz), grid rebuilt at the
 * current positions, with the particles' current densities. */
int ref_vertex_normals(ref_sim* s, const double* posV, int nV, float scale, double* normals) {
    int rc = ref_search(s);
    if (rc) return rc;
    UniformGrid* g = &s->grid;
    launch1d((unsigned)nV, true, [&] {
        computeNormales_Vertexs_Kernel((double3*)posV, (double3*)normals, scale, nV, g->Min, g->sizeCell, g->nbCellsX,
                                       g->nbCellsY, g->nbCellsZ, g->nbParticles, g->indexParticles,
                                       (double3*)s->pos.data(), s->radius.data(), s->mass.data(), s->density.data(), s->n);
    });
    return 0;
}

/* evaluate_ForceExt_Trochoide (ForceExt.cu:37-52) on n particles. */
int ref_force_trochoid(int n, double* pos, double* accum, double* mass, float A, float k, float theta, float w, float phi,
                       float t) {
    launch1d((unsigned)n, true, [&] { evaluate_force_trochoide(n, (double3*)pos, (double3*)accum, mass, A, k, theta, w, phi, t); });
    return 0;
}

/* evaluate_ForceExt_Constante (ForceExt.cu:24-34) on n particles. */
int ref_force_constant(int n, double* accum, double* mass, const float* dir, float amp) {
    const float3 d = make_float3(dir[0], dir[1], dir[2]);
    launch1d((unsigned)n, true, [&] { evaluate_force_constante(n, (double3*)accum, mass, d, amp); });
    return 0;
}

/* createGrid_MarchingCube_CUDA (MarchingCube.cu:12-28): node centres as double4. */
int ref_mc_grid(const double* centre, double l, double w, double d, float cell, int nx, int ny, int nz, double* nodes4) {
    std::vector<int> nb((size_t)nx * ny * nz, 0);
    launch_cells(nx, ny, nz, [&] {
        createGrid_MarchingCube_Kernel((double4*)nodes4, make_double3(centre[0], centre[1], centre[2]), l, w, d, cell,
                                       nx, ny, nz, nb.data());
    });
    return 0;
}

/* SPHSystem::evaluateIso -> evaluateIso_CUDA -> evaluateIso_Kernel
 * (UniformGridKernel.cu:98-138) over the node positions `nodes` (x fastest,
 * nx*ny*nz nodes, xyz), with the grid rebuilt at the current positions.
 * One emulated thread per node. */
int ref_iso(ref_sim* s, const double* nodes, int nx, int ny, int nz, double scale, double* iso) {
    int rc = ref_search(s);
    if (rc) return rc;
    const size_t nn = (size_t)nx * ny * nz;
    std::vector<double4> grid4(nn);
    for (size_t i = 0; i < nn; ++i) grid4[i] = make_double4(nodes[3 * i], nodes[3 * i + 1], nodes[3 * i + 2], 0.0);
    UniformGrid* g = &s->grid;
    launch_cells(nx, ny, nz, [&] {
        evaluateIso_Kernel(grid4.data(), nx, ny, nz, scale, g->Min, g->sizeCell, g->nbCellsX, g->nbCellsY,
                           g->nbCellsZ, g->nbParticles, g->indexParticles, (double3*)s->pos.data(), s->radius.data(),
                           s->n);
    });
    for (size_t i = 0; i < nn; ++i) iso[i] = grid4[i].w;
    return 0;
}

/* polygonize_MarchingCube_CUDA (MarchingCube.cu:31-46) over nodes given as
 * (x, y, z, iso), x fastest. The kernel writes each cell's triangle corners
 * to its own slots (nbVertexMax_perCell per cell); they are returned here in
 * cell order, three per triangle: at most `cap` vertices, the count in *nv. */
int ref_marching_cubes(const double* nodes4, int nx, int ny, int nz, double level, int64_t cap, double* vert,
                       int64_t* nv) {
    const size_t size = (size_t)nx + (size_t)nx * ny + (size_t)nx * ny * nz;   /* MarchingCube.cu's allocation */
    std::vector<double4> grid4((size_t)nx * ny * nz);
    std::memcpy(grid4.data(), nodes4, sizeof(double4) * grid4.size());
    std::vector<int> nb(size, 0), idx(size * nbIndexMax_perCell, 0);
    std::vector<double3> vx(size * nbVertexMax_perCell), nm(size * nbVertexMax_perCell);
    launch_cells(nx, ny, nz, [&] {
        polygonize_MarchingCube_Kernel(grid4.data(), nx, ny, nz, level, nb.data(), vx.data(), nm.data(), idx.data());
    });
    int64_t k = 0;
    for (size_t c = 0; c < size; ++c)
        for (int m = 0; m < nb[c]; ++m, ++k)
            if (k < cap) {
                const double3 p = vx[c * nbVertexMax_perCell + m];
                vert[3 * k] = p.x; vert[3 * k + 1] = p.y; vert[3 * k + 2] = p.z;
            }
    *nv = k;
    return k > cap ? -1 : 0;
}

/* One collision object on n particles, through the launch its reference
 * launcher makes (PlaneCollision.cu:9-21, SphereCollision.cu:9-16 -- its
 * argument order included, CylinderCollision.cu:9-19, MeshCollision.cu:8-18,
 * Linear/Gaussian/PeriodicHeightFieldCollision.cu:9-21). v[] and the layouts
 * of faces (count x 12 floats) and terms (count x 6 doubles) are
 * orc_collider's. A height object is one linear term, one Gaussian term or
 * cosine terms only (the reference's three kernels). */
int ref_collide(int type, int n, double* old_pos, double* pos, double* vel, float dt, float elast, int container,
                float particle_radius, const float* v, int count, const float* faces, const double* terms) {
    if (n <= 0) return 0;
    double3* np = (double3*)pos;
    double3* nv = (double3*)vel;
    double3* op = (double3*)old_pos;
    auto f3 = [](const float* a) { return make_float3(a[0], a[1], a[2]); };
    if (type == 1) {
        launch1d(n, true, [&] { collisionPlan(n, np, nv, op, nv, f3(v), f3(v + 3), f3(v + 6), f3(v + 9), f3(v + 12), elast, dt); });
    } else if (type == 2) {
        const float3 O = f3(v);
        const float radius = v[3];
        const bool cont = container != 0;
        launch1d(n, true, [&] { collisionSphere(n, np, nv, op, nv, O, radius, elast, dt, cont); });
    } else if (type == 3) {
        launch1d(n, true, [&] {
            collisionCylinder(n, np, nv, particle_radius, dt, elast, container != 0, f3(v), v[6], v[7], f3(v + 3));
        });
    } else if (type == 4) {
        std::vector<float> fa(3 * (size_t)count), fb(fa.size()), fc(fa.size()), fn(fa.size());
        for (int f = 0; f < count; ++f)
            for (int a = 0; a < 3; ++a) {
                fa[3 * f + a] = faces[12 * f + a];
                fb[3 * f + a] = faces[12 * f + 3 + a];
                fc[3 * f + a] = faces[12 * f + 6 + a];
                fn[3 * f + a] = faces[12 * f + 9 + a];
            }
        launch1d(n, true, [&] {
            collisionTriangle(n, (uint)count, np, nv, op, nv, fa.data(), fb.data(), fc.data(), fn.data(), elast,
                              particle_radius, dt);
        });
    } else if (type == 5) {
        const float3 mn = f3(v), mx = f3(v + 3);
        const int kind = (int)terms[0];
        if (kind == 1 && count == 1) {
            launch1d(n, true, [&] {
                collisionSystem_Linear_HeightFieldCollision_Kernel(np, nv, particle_radius, dt, n, terms[1], terms[2],
                                                                   mn, mx, elast);
            });
        } else if (kind == 2 && count == 1) {
            launch1d(n, true, [&] {
                collisionSystem_Gaussian_HeightFieldCollision_Kernel(np, nv, particle_radius, dt, n, terms[1],
                                                                     terms[2], terms[3], terms[4], terms[5], mn, mx,
                                                                     elast);
            });
        } else {
            std::vector<double> A(count), k(count), th(count), ph(count);
            for (int i = 0; i < count; ++i) {
                if ((int)terms[6 * i] != 3) return -2;
                A[i] = terms[6 * i + 1]; k[i] = terms[6 * i + 2]; th[i] = terms[6 * i + 3]; ph[i] = terms[6 * i + 4];
            }
            launch1d(n, true, [&] {
                collisionSystem_Periodic_HeightFieldCollision_Kernel(np, nv, particle_radius, dt, n, (uint)count,
                                                                     A.data(), k.data(), th.data(), ph.data(), mn,
                                                                     mx, elast);
            });
        }
    } else {
        return -1;
    }
    return 0;
}

}  /* extern "C" */
