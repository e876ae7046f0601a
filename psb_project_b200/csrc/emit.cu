// emit.cu -- emission into the resident state: particles appended at slots
// (and ids) n0 .. n0 + k - 1 of the current buffers, with density and
// pressure 0. Nothing already resident moves.
#include <cuda_runtime.h>

#include "psb.h"
#include "psb_internal.cuh"
#include "emitters.h"

namespace psb {
namespace {

constexpr int kT = 256;

__device__ __forceinline__ void put(int t, float3 x, float3 v, int dem, float4* pos, float4* vel, float4* vap,
                                    int* ids, float2* rp) {
    pos[t] = make_float4(x.x, x.y, x.z, 0.f);
    vel[t] = make_float4(v.x, v.y, v.z, 0.f);
    vap[t] = dem ? make_float4(v.x, v.y, v.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    ids[t] = t;
    rp[t] = make_float2(0.f, 0.f);
}

// A stored emission (box, sphere, cylinder, heart): xyz holds k positions.
__global__ void __launch_bounds__(kT) k_emit_list(int n0, int k, const float* __restrict__ xyz, float3 v, int dem,
                                                  float4* pos, float4* vel, float4* vap, int* ids, float2* rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    put(n0 + i, make_float3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), v, dem, pos, vel, vap, ids, rp);
}

struct RandomEmitter {
    int type;            // PSB_EMITTER_ELLIPSOID or PSB_EMITTER_MESH
    int count;           // per emission (ellipsoid) or per face (mesh)
    unsigned emission;
    unsigned long long seed;
    float v[12];
    const float* faces;  // mesh: 9 floats per face
};

// A random emission drawn on the device (the same draws as the host's).
__global__ void __launch_bounds__(kT) k_emit_random(int n0, int k, RandomEmitter e, float3 v, int dem, float4* pos,
                                                    float4* vel, float4* vap, int* ids, float2* rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    float x[3];
    if (e.type == PSB_EMITTER_ELLIPSOID) emit::ellipsoid_point(e.v, e.seed, e.emission, (uint64_t)i, x);
    else emit::mesh_point(e.faces + 9 * (size_t)(i / e.count), e.seed, e.emission, (uint64_t)i, x);
    put(n0 + i, make_float3(x[0], x[1], x[2]), v, dem, pos, vel, vap, ids, rp);
}

__global__ void k_append_ids(int n0, int k, int* ids, float2* rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    ids[n0 + i] = n0 + i;
    rp[n0 + i] = make_float2(0.f, 0.f);
}

inline unsigned nblocks(int k) { return (unsigned)((k + kT - 1) / kT); }

}  // namespace

void launch_emit_list(cudaStream_t st, int n0, int k, const float* xyz, const float* v, int dem, float4* pos,
                      float4* vel, float4* vap, int* ids, float2* rp) {
    if (k <= 0) return;
    k_emit_list<<<nblocks(k), kT, 0, st>>>(n0, k, xyz, make_float3(v[0], v[1], v[2]), dem, pos, vel, vap, ids, rp);
}

void launch_emit_random(cudaStream_t st, int n0, int k, int type, int count, unsigned emission,
                        unsigned long long seed, const float* params, const float* faces, const float* v, int dem,
                        float4* pos, float4* vel, float4* vap, int* ids, float2* rp) {
    if (k <= 0) return;
    RandomEmitter e{};
    e.type = type;
    e.count = count;
    e.emission = emission;
    e.seed = seed;
    for (int a = 0; a < 12; ++a) e.v[a] = params[a];
    e.faces = faces;
    k_emit_random<<<nblocks(k), kT, 0, st>>>(n0, k, e, make_float3(v[0], v[1], v[2]), dem, pos, vel, vap, ids, rp);
}

void launch_append_ids(cudaStream_t st, int n0, int k, int* ids, float2* rp) {
    if (k <= 0) return;
    k_append_ids<<<nblocks(k), kT, 0, st>>>(n0, k, ids, rp);
}

}  // namespace psb
