// emitters.h -- the draws of the random emitters (ellipsoid, mesh), shared
// by the host generator (emitters.cpp) and the device emission kernel
// (emit.cu), so that both produce the same particles.
//
// The reference draws with the C library's rand() (EmitterElipsoide.cpp,
// EmitterMesh.cpp seeds it with time(NULL)); here every draw is a function
// of (seed, emission, particle, draw): SplitMix64 (Steele, Lea, Flood 2014)
// over a key that packs the four, 53 bits of it as a double in [0, 1).
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "psb.h"

#ifdef __CUDACC__
#define PSB_HD __host__ __device__
#else
#define PSB_HD
#endif

namespace psb {
namespace emit {

PSB_HD inline uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

PSB_HD inline double uniform(uint64_t seed, uint32_t emission, uint64_t particle, uint32_t draw) {
    const uint64_t k = splitmix64(seed ^ splitmix64(((uint64_t)emission << 32) | draw) ^ splitmix64(particle + 1));
    return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

constexpr double kTwoPi = 6.283185307179586;

// EmitterElipsoide.cpp:33-45: t in [0, 2 pi); offsets x, z uniform over
// [-a/2, a/2] x [-b/2, b/2] (float); the point t on the ellipse scaled by 1/100.
// v: center(3), a, b.
PSB_HD inline void ellipsoid_point(const float* v, uint64_t seed, uint32_t e, uint64_t i, float* out) {
    const double t = uniform(seed, e, i, 0) * kTwoPi;
    const double cx = (double)v[3] * cos(t), cz = (double)v[4] * sin(t);
    const float x = (float)(-v[3] / 2 + uniform(seed, e, i, 1) * v[3]);
    const float z = (float)(-v[4] / 2 + uniform(seed, e, i, 2) * v[4]);
    out[0] = (float)((double)v[0] + x + cx / 100);
    out[1] = v[1];
    out[2] = (float)((double)v[2] + z + cz / 100);
}

// EmitterMesh.cpp:31-42: weights a, b, c uniform in [0, 0.5) (float), the
// point (a A + b B + c C)/(a + b + c). face: A, B, C (9 floats).
PSB_HD inline void mesh_point(const float* face, uint64_t seed, uint32_t e, uint64_t i, float* out) {
    const float a = (float)(uniform(seed, e, i, 0) * 0.5);
    const float b = (float)(uniform(seed, e, i, 1) * 0.5);
    const float c = (float)(uniform(seed, e, i, 2) * 0.5);
    const double s = (double)(a + b + c);
    for (int k = 0; k < 3; ++k)
        out[k] = (float)(((double)a * face[k] + (double)b * face[3 + k] + (double)c * face[6 + k]) / s);
}

// Host: the positions of one emission of e (xyz, stride 3) into pos, at
// most `limit` points. PSB_EINVAL for an emitter whose loops cannot end or
// whose bound passes 2^31 - 1 points, PSB_EOVERFLOW_NBR when the emission has
// more than `limit` points (the generator stops there), PSB_ENOMEM.
int generate(const psb_emitter& e, int32_t emission, int64_t limit, std::vector<float>& pos);

}  // namespace emit
}  // namespace psb
