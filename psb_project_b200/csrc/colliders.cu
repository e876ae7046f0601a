// colliders.cu -- collision objects after the integrator (native path) and
// the reference's collision launchers on its own FP64 AoS buffers
// (include/psb_compat.h). The per-object formulas are in colliders.cuh.
//
// Native: WCSPH and DEM steps write their output to the other state buffer,
// so the objects run as one extra elementwise sweep that reads the start
// positions from the input buffer; the PCISPH commit applies them inline
// (k_pci_commit). Objects act in list order, after the box walls.
//
// Compat: one launch per object, as the reference's ObjectCollision
// subclasses issue them (Collision.cpp:44-49), synchronous like its
// launchers; the state is FP64 and the arithmetic the reference performs in
// float stays float.
#include <cuda_runtime.h>
#include <cmath>

#include "psb_internal.cuh"
#include "colliders.cuh"
#include "psb_compat.h"

namespace psb {
namespace {

constexpr int kT = 256;
inline unsigned nblocks(long long n) { return (unsigned)((n + kT - 1) / kT); }

using coll::V3;

__global__ void __launch_bounds__(kT) k_apply_colliders(Params P, const float4* __restrict__ x_old,
                                                        const float4* __restrict__ vh_old, float4* __restrict__ pos,
                                                        float4* __restrict__ vel, float4* __restrict__ vap) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xo = x_old[t], xn = pos[t];
    const float4 vn = vh_old ? vap[t] : vel[t];
    V3<float> x{xn.x, xn.y, xn.z}, v{vn.x, vn.y, vn.z};
    coll::apply_colliders(P.coll, P.n_coll, P.dt, V3<float>{xo.x, xo.y, xo.z}, x, v);
    pos[t] = make_float4(x.x, x.y, x.z, xn.w);
    vap[t] = make_float4(v.x, v.y, v.z, 0.f);
    if (vh_old) {
        const float4 vh = vh_old[t];
        vel[t] = make_float4((vh.x + v.x) * 0.5f, (vh.y + v.y) * 0.5f, (vh.z + v.z) * 0.5f, 0.f);
    } else {
        vel[t] = make_float4(v.x, v.y, v.z, 0.f);
    }
}

// ---- compat: FP64 state ------------------------------------------------------
__device__ __forceinline__ V3<double> ld(const double* a, long long i) {
    return V3<double>{a[3 * i], a[3 * i + 1], a[3 * i + 2]};
}
__device__ __forceinline__ void st(double* a, long long i, V3<double> v) {
    a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z;
}

// Plane, sphere, cylinder and mesh objects; old_pos may be null for the
// objects that do not read it (sphere, cylinder).
__global__ void k_collide_compat(Collider o, float dt, int n, const double* __restrict__ old_pos,
                                 double* __restrict__ new_pos, double* __restrict__ new_vel) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<double> xo = old_pos ? ld(old_pos, i) : V3<double>{0, 0, 0};
    V3<double> x = ld(new_pos, i), v = ld(new_vel, i);
    bool hit = false;
    switch (o.type) {
        case COLL_PLANE: hit = coll::plane<double>(o, dt, xo, x, v); break;
        case COLL_SPHERE: hit = coll::sphere<double>(o, dt, xo, x, v); break;
        case COLL_CYLINDER: hit = coll::cylinder<double>(o, dt, xo, x, v); break;
        case COLL_MESH: hit = coll::mesh<double>(o, dt, xo, x, v); break;
        default: break;
    }
    if (hit) {
        st(new_pos, i, x);
        st(new_vel, i, v);
    }
}

// Height functions of the reference's three height-field collision kernels,
// in FP64 (the Gaussian's squares go through powf there, so float here).
struct LinearH {
    double a, b;   // LinearHeightFieldCollision_Kernel.cu:11-14
    __device__ double operator()(double x, double z) const { return a * x + b * z; }
};
struct GaussianH {
    double A, x0, z0, p1, p2;   // GaussianHeightFieldCollision_Kernel.cu:10-13
    __device__ double operator()(double x, double z) const {
        return A * exp(-((double)coll::fsq((float)(x - x0)) / (2 * p1 * p1) +
                         (double)coll::fsq((float)(z - z0)) / (2 * p2 * p2)));
    }
};
struct PeriodicH {
    unsigned nf;   // PeriodicHeightFieldCollision_Kernel.cu:10-16
    const double *A, *k, *theta, *phi;
    __device__ double operator()(double x, double z) const {
        double y = 0;
        for (unsigned i = 0; i < nf; ++i) y += A[i] * cos(k[i] * (x * cos(theta[i]) + z * sin(theta[i])) + phi[i]);
        return y;
    }
};

template <class H>
__global__ void k_height_compat(Collider o, float dt, int n, H h, double* __restrict__ new_pos,
                                double* __restrict__ new_vel) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<double> x = ld(new_pos, i), v = ld(new_vel, i);
    if (coll::height<double>(o, dt, x, v, h)) {
        st(new_pos, i, x);
        st(new_vel, i, v);
    }
}

inline void put3(float* dst, psb_vec3 a) {
    dst[0] = (float)a.e[0]; dst[1] = (float)a.e[1]; dst[2] = (float)a.e[2];
}

Collider blank(int type, float elast) {
    Collider o{};
    o.type = type;
    o.elast = elast;
    return o;
}

Collider footprint(psb_vec3 mn, psb_vec3 mx, float elast) {
    Collider o = blank(COLL_HEIGHT, elast);
    put3(o.v, mn);
    put3(o.v + 3, mx);
    return o;
}

}  // namespace

void launch_apply_colliders(cudaStream_t st, const Params& P, const float4* x_old, const float4* vh_old, float4* pos,
                            float4* vel, float4* vap) {
    if (P.n <= 0 || P.n_coll <= 0) return;
    k_apply_colliders<<<nblocks(P.n), kT, 0, st>>>(P, x_old, vh_old, pos, vel, vap);
}

}  // namespace psb

using psb::Collider;

extern "C" {

void collisionPlan_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, psb_vec3 A, psb_vec3 B,
                        psb_vec3 C, psb_vec3 D, psb_vec3 N, float elast, float dt, int nbBodiesP) {
    (void)oldVel;
    if (nbBodiesP <= 0) return;
    Collider o = psb::blank(psb::COLL_PLANE, elast);
    psb::put3(o.v, A); psb::put3(o.v + 3, B); psb::put3(o.v + 6, C); psb::put3(o.v + 9, D); psb::put3(o.v + 12, N);
    psb::k_collide_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(o, dt, nbBodiesP, oldPos, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionSystem_Sphere_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle,
                                 float dt, int nbBodies, psb_vec3 origin, float radius, float elast, bool container) {
    (void)oldPos; (void)oldVel; (void)radiusParticle;
    if (nbBodies <= 0) return;
    Collider o = psb::blank(psb::COLL_SPHERE, elast);
    psb::put3(o.v, origin);
    o.v[3] = radius;
    o.flag = container ? 1 : 0;
    psb::k_collide_compat<<<psb::nblocks(nbBodies), psb::kT>>>(o, dt, nbBodies, nullptr, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionCylinder_CUDA(double* newPos, double* newVel, float radiusParticle, float dt, int nbBodiesP,
                            psb_vec3 center, psb_vec3 direction, double radius, double length, float elast,
                            bool container) {
    (void)radiusParticle; (void)elast; (void)container;
    if (nbBodiesP <= 0) return;
    Collider o = psb::blank(psb::COLL_CYLINDER, 0.3f);
    psb::put3(o.v, center);
    psb::put3(o.v + 3, direction);
    o.v[6] = (float)radius;
    o.v[7] = (float)length;
    psb::k_collide_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(o, dt, nbBodiesP, nullptr, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionMesh_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel, float radiusParticle, float dt,
                        unsigned int nbFaces, float* fA, float* fB, float* fC, float* fN, float elast, int nbBodiesP) {
    (void)oldVel; (void)radiusParticle; (void)elast;
    if (nbBodiesP <= 0 || nbFaces == 0) return;
    Collider o = psb::blank(psb::COLL_MESH, 0.f);
    o.count = (int)nbFaces;
    o.fa = fA; o.fb = fB; o.fc = fC; o.fn = fN;
    o.stride = 3;
    psb::k_collide_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(o, dt, nbBodiesP, oldPos, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionSystem_Linear_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel, double* newVel,
                                                      double radiusParticle, float dt, unsigned int nbBodiesP,
                                                      double a, double b, psb_vec3 Min, psb_vec3 Max, float elast) {
    (void)oldPos; (void)oldVel; (void)radiusParticle;
    if (nbBodiesP == 0) return;
    psb::k_height_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(psb::footprint(Min, Max, elast), dt, (int)nbBodiesP,
                                                               psb::LinearH{a, b}, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionSystem_Gaussian_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, double A, double x0, double z0,
                                                        double p1, double p2, psb_vec3 Min, psb_vec3 Max,
                                                        float elast) {
    (void)oldPos; (void)oldVel; (void)radiusParticle;
    if (nbBodiesP == 0) return;
    psb::k_height_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(psb::footprint(Min, Max, elast), dt, (int)nbBodiesP,
                                                               psb::GaussianH{A, x0, z0, p1, p2}, newPos, newVel);
    cudaDeviceSynchronize();
}

void collisionSystem_Periodic_HeightFieldCollision_CUDA(double* oldPos, double* newPos, double* oldVel,
                                                        double* newVel, double radiusParticle, float dt,
                                                        unsigned int nbBodiesP, unsigned int nbFunc, double* A,
                                                        double* k, double* theta, double* phi, psb_vec3 Min,
                                                        psb_vec3 Max, float elast) {
    (void)oldPos; (void)oldVel; (void)radiusParticle;
    if (nbBodiesP == 0) return;
    psb::k_height_compat<<<psb::nblocks(nbBodiesP), psb::kT>>>(psb::footprint(Min, Max, elast), dt, (int)nbBodiesP,
                                                               psb::PeriodicH{nbFunc, A, k, theta, phi}, newPos,
                                                               newVel);
    cudaDeviceSynchronize();
}

}  // extern "C"
