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
 * reference's order (UniformGrid.cuh:16-33, SphKernel.cuh:6-10), and
 * psb_vec3 has the layout of the reference's Vector3 (Vector3.h: one
 * double e[3], no virtual members), which its callers pass by value.
 *
 * Not provided: evaluate_ForceExt_Constante / _Trochoide (they take the
 * reference's ForceExt class objects; the scene's gravity replaces them),
 * evaluate_densities_forces, evaluateIso_CUDA and the marching-cubes
 * launchers (psb_iso_field / psb_extract_surface in psb.h replace them).
 */
#ifndef PSB_COMPAT_H
#define PSB_COMPAT_H
#include <stdbool.h>
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

typedef struct {
    double e[3];
} psb_vec3;

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
                              int nbBodiesP, psb_vec3 Min, psb_vec3 Max, bool container, float elast);
/* The other collision objects, on (oldPos, newPos, newVel) in FP64 with the
 * float arithmetic of their kernels (the formulas and the behaviours they
 * keep are those of psb_set_colliders in psb.h):
 * PlaneCollision.cu:9-21 / PlaneCollision_Kernel.cu:7-81 */
void collisionPlan_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, psb_vec3 A, psb_vec3 B,
                        psb_vec3 C, psb_vec3 D, psb_vec3 N, float elast, float dt, int nbBodiesP);
/* SphereCollision.cu:9-16 / SphereCollision_Kernel.cu:7-91 */
void collisionSystem_Sphere_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle,
                                 float dt, int nbBodies, psb_vec3 origin, float radius, float elast, bool container);
/* CylinderCollision.cu:9-19 / CylinderCollision_Kernel.cu:4-103 */
void collisionCylinder_CUDA(double* newPos, double* newVel, float radiusParticle, float dt, int nbBodiesP,
                            psb_vec3 center, psb_vec3 direction, double radius, double length, float elast,
                            bool container);
/* MeshCollision.cu:8-18 / MeshCollision_Kernel.cu:14-137: fA, fB, fC, fN are
 * device float arrays of 3 nbFaces (corners and normals) */
void collisionMesh_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                        unsigned int nbFaces, float* fA, float* fB, float* fC, float* fN, float elast, int nbBodiesP);
/* LinearHeightFieldCollision.cu:9-20: h = a x + b z */
void collisionSystem_Linear_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                      double radiusParticle, float dt, unsigned int nbBodiesP,
                                                      double a, double b, psb_vec3 Min, psb_vec3 Max, float elast);
/* GaussianHeightFieldCollision.cu:9-21: h = A exp(-((x-x0)^2/(2 p1^2) + (z-z0)^2/(2 p2^2))) */
void collisionSystem_Gaussian_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, double A, double x0, double z0,
                                                        double p1, double p2, psb_vec3 Min, psb_vec3 Max,
                                                        float elast);
/* PeriodicHeightFieldCollision.cu:9-21: h = sum_i A_i cos(k_i (x cos theta_i
 * + z sin theta_i) + phi_i), the four arrays on the device */
void collisionSystem_Periodic_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, unsigned int nbFunc, double* A,
                                                        double* k, double* theta, double* phi, psb_vec3 Min,
                                                        psb_vec3 Max, float elast);
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

#ifdef __cplusplus
}
#endif
#endif /* PSB_COMPAT_H */
