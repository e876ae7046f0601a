/*
 * psb_compat.h -- the reference's extern "C" launchers under their own names
 * and signatures, implemented on the B200 library (libpsb.so), so that the
 * reference's system classes link unchanged.
 *
 * Every function takes the reference's device buffers (AoS double3, per-
 * particle parameter arrays, UniformGrid, partVoisine), returns void and is
 * synchronous, as the reference's launchers are. Where the reference writes
 * out of bounds (more than 64 particles in a cell, more than 200 neighbours)
 * these clamp, print one line to stderr and keep going. The primary
 * interface is psb.h; this layer converts at the call boundary.
 *
 * Types: UniformGrid and partVoisine have the reference's members in the
 * reference's order (UniformGrid.cuh:16-33, SphKernel.cuh:6-10). psb_vec3
 * has the layout of the reference's Vector3 (Vector3.h: one double e[3], no
 * virtual members) and, in C++, a user-provided copy constructor as
 * Vector3 has: the Itanium C++ ABI then passes it "by value" through a
 * hidden pointer to a temporary, so a Vector3 argument of the reference's
 * callers arrives intact. C callers pass that pointer themselves
 * (psb_vec3_arg is const psb_vec3* in C). The external-force launchers
 * take the reference's ForceExt_Constante / ForceExt_Trochoide objects and
 * read their members through the Itanium layout of those classes (a
 * vtable pointer for ForceExt's virtual draw(), then the members in
 * declaration order: Vector3 direction and float amplitude; floats A,
 * lambda, k, theta, w, f, phi, time).
 *
 * With these, every launcher the reference's SPHSystem, PCI_SPHSystem,
 * CudaSystem, SimpleSystem and SurfaceSPH call resolves in libpsb.so.
 */
#ifndef PSB_COMPAT_H
#define PSB_COMPAT_H
#include <stdbool.h>
#include <stddef.h>
#include <vector_types.h>   /* float3, double3 */

#ifdef __cplusplus
extern "C" {
#endif

#ifndef PSB_COMPAT_MAXPARTICLES
#define PSB_COMPAT_MAXPARTICLES 64     /* slots per cell, UniformGrid.cuh:8 */
#endif
#define PSB_COMPAT_MAX_NEIGHBOURS 200  /* listeVoisine stride, UniformGridKernel.cu:84 */

typedef struct {
    int* nbVoisines;
    int* listeVoisine;
} partVoisine;

typedef struct {
    float3 Min;
    float3 Max;
    float sizeCell;
    double l, h, d;
    int* indexParticles;
    int* nbParticles;
    double3* m_dPos;
    double* m_hPos;
    float* m_dIsoVal;
    float* m_hIsoVal;
    float* m_dIsoNorm;
    float* m_hIsoNorm;
    int nbCellsX;
    int nbCellsY;
    int nbCellsZ;
} UniformGrid;

typedef struct psb_vec3 {
    double e[3];
#ifdef __cplusplus
    psb_vec3() : e{0, 0, 0} {}
    psb_vec3(double x, double y, double z) : e{x, y, z} {}
    psb_vec3(const psb_vec3& v) : e{v.e[0], v.e[1], v.e[2]} {}    /* user-provided, as Vector3's */
    psb_vec3& operator=(const psb_vec3& v) = default;
#endif
} psb_vec3;
#ifdef __cplusplus
typedef psb_vec3 psb_vec3_arg;          /* non-trivial for calls: passed through a hidden pointer */
class ForceExt_Constante;               /* the reference's classes (ForceExt_Constante.h, ForceExt_Trochoide.h) */
class ForceExt_Trochoide;
#else
typedef const psb_vec3* psb_vec3_arg;   /* the same calling convention, spelled out for C */
typedef struct ForceExt_Constante ForceExt_Constante;
typedef struct ForceExt_Trochoide ForceExt_Trochoide;
#endif
struct cudaGraphicsResource;
#define PSB_COMPAT_MC_SLOTS 200          /* vertex and index slots per marching-cubes cell, MarchingCube.cuh:13-15 */

/* UniformGrid.cu:17-44: Min = C - L/2, cells = ceil(L/sizeCell), device
 * arrays for slots, counts and cell centres. */
void createGrid(double xC, double yC, double zC, double length, double width, double depth, float sizeCell,
                UniformGrid* grid);
/* UniformGrid.cu:53-60 */
void _finalizeGrid(UniformGrid* grid);
/* UniformGrid.cu:64-76: every cell count to 0 */
void reinitCells(UniformGrid* grid);
/* UniformGrid.cu:80-87 / UniformGridKernel.cu:43-55: particle p goes to cell
 * floor((x - Min)/sizeCell) (FP64 from the float Min and sizeCell), in the
 * next free slot */
void storeParticles(UniformGrid* grid, double* pos, unsigned int nbBodies);
/* UniformGrid.cu:91-98 / UniformGridKernel.cu:58-95: j is listed for i when
 * length(x_i - x_j) <= radius[i] within ceil(scale) cell rings (self
 * included), in cell-walk and slot order */
void searchNeighbooring(double* pos, double* radius, UniformGrid* grid, double scale, partVoisine voisines,
                        unsigned int nbBodies);

/* SphSystem.cu:6-14 / SphKernel.cu:112-124: leap-frog v- = v+, v+ += F/rho dt,
 * x_old = x, x += v+ dt */
void integrateSPHSystem(double* velInterAv, double* velInterAp, double* oldPos, double* newPos, double* forces,
                        double* densities, double dt, int numBodies);
/* SphSystem.cu:17-24 / SphKernel.cu:128-135: v_old = v, v = (v- + v+)/2 */
void interpolateSPHVelocities(double* velInterAv, double* velInterAp, double* oldVel, double* newVel, int numBodies);
/* System.cu:6-12 / ParticleKernel.cu:12-20: v += F/m dt, x += v_old dt on (newPos, newVel) */
void integrateSystem(double* oldPos, double* newPos, double* oldVel, double* newVel, double* forces, double* mass,
                     double dt, int start, int numBodies);
/* CudaSystem.cu:6-14 / CudaParticle_Kernel.cu:10-55: adds to forces[A] the
 * contact forces of A's listed neighbours as the reference executes them:
 * -spring (R - d) n with R = r_A + r_B, d < 2R (its damping, shear and
 * attraction terms go through a double3 operator+= that does not assign) */
void interactionSystem(double* oldPos, double* oldVel, double* forces, double* interactionRadius, double* spring,
                       double* damping, double* shear, double* attraction, partVoisine voisines, int numBodies);
/* BoxCollision.cu:10-18 / BoxCollision_Kernel.cu:7-34: clamp into
 * [Min + r, Max - r], remove the velocity along the summed wall normals */
void collisionSystem_Box_CUDA(double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                              int nbBodiesP, psb_vec3_arg Min, psb_vec3_arg Max, bool container, float elast);
/* The other collision objects, on (oldPos, newPos, newVel) in FP64 with the
 * float arithmetic of their kernels (the formulas and the behaviours they
 * keep are those of psb_set_colliders in psb.h):
 * PlaneCollision.cu:9-21 / PlaneCollision_Kernel.cu:7-81 */
void collisionPlan_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, psb_vec3_arg A, psb_vec3_arg B,
                        psb_vec3_arg C, psb_vec3_arg D, psb_vec3_arg N, float elast, float dt, int nbBodiesP);
/* SphereCollision.cu:9-16 / SphereCollision_Kernel.cu:7-91 */
void collisionSystem_Sphere_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle,
                                 float dt, int nbBodies, psb_vec3_arg origin, float radius, float elast, bool container);
/* CylinderCollision.cu:9-19 / CylinderCollision_Kernel.cu:4-103 */
void collisionCylinder_CUDA(double* newPos, double* newVel, float radiusParticle, float dt, int nbBodiesP,
                            psb_vec3_arg center, psb_vec3_arg direction, double radius, double length, float elast,
                            bool container);
/* MeshCollision.cu:8-18 / MeshCollision_Kernel.cu:14-137: fA, fB, fC, fN are
 * device float arrays of 3 nbFaces (corners and normals) */
void collisionMesh_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                        unsigned int nbFaces, float* fA, float* fB, float* fC, float* fN, float elast, int nbBodiesP);
/* LinearHeightFieldCollision.cu:9-20: h = a x + b z */
void collisionSystem_Linear_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                      double radiusParticle, float dt, unsigned int nbBodiesP,
                                                      double a, double b, psb_vec3_arg Min, psb_vec3_arg Max, float elast);
/* GaussianHeightFieldCollision.cu:9-21: h = A exp(-((x-x0)^2/(2 p1^2) + (z-z0)^2/(2 p2^2))) */
void collisionSystem_Gaussian_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, double A, double x0, double z0,
                                                        double p1, double p2, psb_vec3_arg Min, psb_vec3_arg Max,
                                                        float elast);
/* PeriodicHeightFieldCollision.cu:9-21: h = sum_i A_i cos(k_i (x cos theta_i
 * + z sin theta_i) + phi_i), the four arrays on the device */
void collisionSystem_Periodic_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, unsigned int nbFunc, double* A,
                                                        double* k, double* theta, double* phi, psb_vec3_arg Min,
                                                        psb_vec3_arg Max, float elast);
/* PciSphSystem.cu:8-68: density, non-pressure forces, three pressure
 * corrections and the final leap-frog with the reference's formulas, run by
 * the B200 kernels (psb_step, reference profile) on a context that this
 * layer keeps per process: pos, oldPos, velInterAv, velInterAp, density and
 * pressure are written as the reference writes them; the neighbour lists
 * are rebuilt with the same test (voisines is not read), and the
 * intermediate buffers (restore_*, normales, force*, densityError) are not
 * written. Parameters are those of particle 0. */
void pci_SPH_update(double* oldPos, double* pos, double* vel, double* velInterAv, double* velInterAp,
                    double* restore_oldPos, double* restore_pos, double* restore_velInterAv,
                    double* restore_velInterAp, double* mass, double* radius, double* density, double* restDensity,
                    double* densityError, double* pressure, double* k, double* viscosity, double* l,
                    double* surfaceTension, double threshold, partVoisine voisines, double* normales,
                    double* forceViscosity, double* forceSurface, double* forcePressure, double* forceAccum, float dt,
                    unsigned int nbBodies);

/* SphSystem.cu:27-43 / SphKernel.cu:9-91: WCSPH density and EOS p = k (rho -
 * rho0) over the 200-slot lists, then the pressure, viscosity and surface-
 * tension force densities, the normals and their sum in forcesAccum */
void evaluate_densities_forces(double* pos, double* vel, double* mass, double* radius, double* densities,
                               double* pressure, double* normales, double* restDensities, double* viscosities,
                               double* k, double* threshold, double* surfaceTension, int numBodies, double* fPressure,
                               double* fViscosity, double* fSurface, double* forcesAccum, partVoisine voisines);
/* ForceExt.cu:24-34 / ForceExt_Constante.cu:15-23: accum += (direction
 * amplitude) mass, direction and amplitude read from the object as floats */
void evaluate_ForceExt_Constante(unsigned int nbBodies, double* accumForceBuffer, double* mass,
                                 ForceExt_Constante* FC);
/* ForceExt.cu:37-52 / ForceExt_Trochoide.cu:14-24: accum.y += A cos(k (x cos
 * theta + z sin theta) w t + phi) mass */
void evaluate_ForceExt_Trochoide(unsigned int nbBodies, double* oldPos, double* accumForceBuffer, double* mass,
                                 ForceExt_Trochoide* T);
/* UniformGrid.cu:102-117 / UniformGridKernel.cu:98-138: posMC is one double4
 * per node (x, y, z, value); the value becomes sum (1/r^6)(r^2 - d^2)^3 over
 * the particles within r = h/scale in floor(1/scale) cell rings (terms in
 * float). Scales below 1/16 (a ring of more than 16 cells) are refused. */
void evaluateIso_CUDA(double* posMC, unsigned int nbCellsX_MC, unsigned int nbCellsY_MC, unsigned int nbCellsZ_MC,
                      double scale, UniformGrid* grid, double* pos, double* radius, unsigned int nbBodies);
/* UniformGrid.cu:120-131 / UniformGridKernel.cu:141-190: -grad c / |grad c|
 * at each vertex over two cell rings */
void computeNormales_Vertex_CUDA(double* posV, double* normales, float scale, unsigned int nbV, UniformGrid* grid,
                                 double* pos, double* radius, double* mass, double* densities, unsigned int nbBodies);
/* MarchingCube.cu:12-28 / MarchingCube_Kernel.cu:14-33: node centres (double4,
 * value 0) and per-cell vertex counts 0 */
void createGrid_MarchingCube_CUDA(psb_vec3_arg C, double l, double w, double d, float sizeCell, unsigned int nbPosX,
                                  unsigned int nbPosY, unsigned int nbPosZ, double* grid, int* m_nbIndex);
/* MarchingCube.cu:32-46 / MarchingCube_Kernel.cu:36-155: per cube (the node
 * at its lowest corner) the triangles of its case, three vertices each,
 * appended to the cube's PSB_COMPAT_MC_SLOTS slots of m_vertex (double3) with
 * m_index[slot] = slot and m_nbIndex counting them. The case table is
 * generated (psb_project_b200/csrc/mc.cu): the same vertices and triangle
 * count per cube as the reference's, a loop may be split into triangles
 * differently. m_normales is not written (nor is it there). */
void polygonize_MarchingCube_CUDA(double* grid, unsigned int nbPosX, unsigned int nbPosY, unsigned int nbPosZ,
                                  double isoLevel, int* m_nbIndex, double* m_vertex, double* m_normales, int* m_index);
/* UniformGrid.cu:135-170 draws the grid with OpenGL: a no-op here (headless). */
void displayGrid(UniformGrid* grid);

/* common.cuh / common.cu:14-107: device count (0: none, -1: driver too old),
 * device set-up (GL interop is not set up: headless), allocation, copies,
 * synchronisation, launch sizing (256 threads; 0 blocks for 0 items) */
int getCudaEnabledDeviceCount(void);
int getcudaEnabledDeviceCount(void);
bool cudaInit(int argc, char** argv);
void cudaGLInit(int argc, char** argv);
void allocateArray(void** devPtr, size_t size);
void freeArray(void* devPtr);
void threadSync(void);
void copyArrayToDevice(void* device, const void* host, int offset, int size);
void copyArrayDeviceToDevice(void* device, const void* host, int offset, int size);
void copyArrayFromDevice(void* host, const void* device, struct cudaGraphicsResource** cuda_vbo_resource, int size);
int iDivUp(int a, int b);
#ifdef __cplusplus
void computeGridSize(int n, int& numBlocks, int& numThreads);
#else
void computeGridSize(int n, int* numBlocks, int* numThreads);
#endif

#ifdef __cplusplus
}
#endif
#endif /* PSB_COMPAT_H */
