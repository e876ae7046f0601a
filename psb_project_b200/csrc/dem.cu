// dem.cu -- the discrete-element step (PSB_DEM): spheres with pairwise
// spring-dashpot contacts over the grid's neighbour lists, gravity, Euler
// integration and the box, in one sweep per step.
//
// Reference profile: CudaSystem::update (CudaSystem.cpp:207-224). Forces are
// m g (evaluate_force_constante, ForceExt_Constante.cu:15-23) plus, for each
// listed neighbour B of A, collideParticle (CudaParticle_Kernel.cu:10-36):
// with rel = x_B - x_A, d = |rel|, R = h_A + h_B (the interaction radius is
// what interactionSystem passes as the sphere radius, CudaSystem.cpp:244),
// and d < 2R:  F += -k_s (R - d) n. The source also adds a dashpot, a shear
// and an attraction term, each as `force += ...`; the reference's double3
// operator+= (double3.h:115-117) returns the sum without assigning it, so
// they never reach the force, and this profile reproduces that.
// integrateEuler (ParticleKernel.cu:12-20): v += F/m dt, x += v_old dt; then
// collisionBox on (x, v).
// Config profile: linear spring-dashpot on overlaps of particle_radius
// spheres, F_A = (-k_n delta + c_n (v_B - v_A).n) n, delta = 2r - d > 0;
// semi-implicit Euler (x += v_new dt); the box.
#include "psb_internal.cuh"

namespace psb {

namespace {

__device__ __forceinline__ void project_box(const Params& P, float3& x, float3& v) {
    // collisionBox (BoxCollision_Kernel.cu:7-34), restitution 0
    float3 pI = x, nI = make_float3(0.f, 0.f, 0.f);
    if (x.x >= P.whi_x) { pI.x = P.whi_x; nI.x = -1.f; }
    if (x.y >= P.whi_y) { pI.y = P.whi_y; nI.y = -1.f; }
    if (x.z >= P.whi_z) { pI.z = P.whi_z; nI.z = -1.f; }
    if (x.x <= P.wlo_x) { pI.x = P.wlo_x; nI.x = 1.f; }
    if (x.y <= P.wlo_y) { pI.y = P.wlo_y; nI.y = 1.f; }
    if (x.z <= P.wlo_z) { pI.z = P.wlo_z; nI.z = 1.f; }
    const float l2 = nI.x * nI.x + nI.y * nI.y + nI.z * nI.z;
    if (l2 > 0.f) {
        const float il = rsqrtf(l2);
        nI.x *= il; nI.y *= il; nI.z *= il;
        const float vd = v.x * nI.x + v.y * nI.y + v.z * nI.z;
        x = pI;
        v.x -= vd * nI.x; v.y -= vd * nI.y; v.z -= vd * nI.z;
    }
}

// STEP false: only the force without the external one (gravity and the
// contacts), written to force; nothing moves.
template <bool REF, bool STEP = true>
__global__ void __launch_bounds__(kBlock) k_dem_step(Params P, const float4* __restrict__ pos,
                                                     const float4* __restrict__ vel, const int* __restrict__ counts,
                                                     const int* __restrict__ list, float4* __restrict__ pos_out,
                                                     float4* __restrict__ vel_out, float4* __restrict__ vap_out,
                                                     float4* __restrict__ force) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xa = pos[t], va = vel[t];
    float3 f = make_float3(P.gx * P.dem_mass, P.gy * P.dem_mass, P.gz * P.dem_mass);
    const int cnt = min(counts[t], P.cap);
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        const float4 xb = pos[j];
        const float rx = xb.x - xa.x, ry = xb.y - xa.y, rz = xb.z - xa.z;
        const float d2 = rx * rx + ry * ry + rz * rz;
        if (!(d2 > 0.f)) return;
        const float rinv = rsqrtf(d2);
        const float d = d2 * rinv;
        if (!(d < P.dem_range)) return;
        const float nx = rx * rinv, ny = ry * rinv, nz = rz * rinv;
        if (REF) {
            // -k_s (R - d) n only: the dashpot, shear and attraction lines of
            // collideParticle are `force += ...` through double3's operator+=,
            // which returns the sum without assigning it (double3.h:115-117)
            const float sn = -P.dem_k * (P.dem_R - d);
            f.x += sn * nx; f.y += sn * ny; f.z += sn * nz;
        } else {
            const float4 vb = vel[j];
            const float vn = (vb.x - va.x) * nx + (vb.y - va.y) * ny + (vb.z - va.z) * nz;
            const float s = -P.dem_k * (P.dem_R - d) + P.dem_c * vn;
            f.x += s * nx; f.y += s * ny; f.z += s * nz;
        }
    });
    if constexpr (!STEP) {
        force[t] = make_float4(f.x, f.y, f.z, 0.f);
        return;
    }
    if (P.ext_force) {      // e.g. the fluid's reaction in a coupled run
        const float4 e = P.ext_force[P.slot_ids[t]];
        f.x += e.x; f.y += e.y; f.z += e.z;
    }
    const float im = P.dem_inv_mass;
    float3 v = make_float3(va.x + f.x * im * P.dt, va.y + f.y * im * P.dt, va.z + f.z * im * P.dt);
    const float3 vx = REF ? make_float3(va.x, va.y, va.z) : v;
    float3 x = make_float3(xa.x + vx.x * P.dt, xa.y + vx.y * P.dt, xa.z + vx.z * P.dt);
    project_box(P, x, v);
    pos_out[t] = make_float4(x.x, x.y, x.z, 0.f);
    vel_out[t] = make_float4(v.x, v.y, v.z, 0.f);
    vap_out[t] = make_float4(v.x, v.y, v.z, 0.f);
    force[t] = make_float4(f.x, f.y, f.z, 0.f);
}

inline int grid_of(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_dem_step(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                     const int* list, float4* pos_out, float4* vel_out, float4* vap_out, float4* force) {
    if (P.n <= 0) return;
    if (P.ref)
        k_dem_step<true><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, counts, list, pos_out, vel_out, vap_out, force);
    else
        k_dem_step<false><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, counts, list, pos_out, vel_out, vap_out, force);
}

void launch_dem_forces(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                       const int* list, float4* force) {
    if (P.n <= 0) return;
    if (P.ref)
        k_dem_step<true, false><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, counts, list, nullptr, nullptr, nullptr,
                                                                 force);
    else
        k_dem_step<false, false><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, counts, list, nullptr, nullptr, nullptr,
                                                                  force);
}

}  // namespace psb
