// scene.cpp -- host-side synthetic scene generator (psb_lattice in psb.h).
//
// Stands in for the reference's EmitterBox lattice emitter
// (src/Kernel/Emitters/EmitterBox.cpp:29-47). The jitter comes from
// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), keyed by seed ^ (3*id + axis) so that every
// particle's position depends only on its id: any subset of a scene can be
// regenerated exactly. Compiled without FMA contraction; the test-suite
// checks it bit for bit against an independent implementation.
#include <cstdint>
#include "psb.h"

namespace {
inline uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
}  // namespace

extern "C" int psb_lattice(const int32_t nxyz[3], double spacing, const double origin[3], double jitter, uint64_t seed,
                           int32_t id0, float* pos) {
    if (!nxyz || !origin || !pos || nxyz[0] <= 0 || nxyz[1] <= 0 || nxyz[2] <= 0 || !(spacing > 0)) return PSB_EINVAL;
    const int64_t nx = nxyz[0], ny = nxyz[1], nz = nxyz[2];
    const int64_t n = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < n; ++id) {
        const int64_t c[3] = {id % nx, (id / nx) % ny, id / (nx * ny)};
        for (int a = 0; a < 3; ++a) {
            const uint64_t z = splitmix64(seed ^ ((uint64_t)(id + id0) * 3u + (uint64_t)a));
            const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);   // 53 bits -> [0, 1)
            const double j = jitter * (2.0 * u - 1.0);
            pos[3 * id + a] = (float)(origin[a] + ((double)c[a] + 0.5) * spacing + j);
        }
    }
    (void)nz;
    return PSB_OK;
}
