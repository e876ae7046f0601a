// emitters.cpp -- host generator of the reference's emitters
// (src/Kernel/Emitters/*): the positions one emission produces.
//
// The deterministic emitters (box, sphere, cylinder, heart) produce the same
// positions at every emission, since none of them moves; the context keeps
// that list on the device and replays it (emit.cu). Their loops follow the
// reference's emitParticles with its types: the box in float, the others in
// double with the C library's sqrt, acos, cos, sin and powf, as the
// reference computes them on the host.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "psb.h"
#include "emitters.h"

namespace {

void push(std::vector<float>& out, double x, double y, double z) {
    out.push_back((float)x);
    out.push_back((float)y);
    out.push_back((float)z);
}

// EmitterBox.cpp:29-47
void box(const psb_emitter& e, std::vector<float>& out) {
    const double cx = e.v[0], cy = e.v[1], cz = e.v[2];
    const float sx = e.v[3], sy = e.v[4], sz = e.v[5];
    const double wx = e.v[6], wy = e.v[7], wz = e.v[8];
    const float step = e.particle_radius * 2;
    for (float z = (float)(cz - sz / 2); (double)z <= cz + sz / 2; z += step)
        for (float y = (float)(cy - sy / 2); (double)y <= cy + sy / 2; y += step)
            for (float x = (float)(cx - sx / 2); (double)x <= cx + sx / 2; x += step) {
                const float dx = (float)(x + wx), dy = (float)(y + wy), dz = (float)(z + wz);
                push(out, dx, dy, dz);
            }
}

// One ring of radius r at height y: angles 0, dt, 2 dt, ... while <= 2 pi
// (EmitterSphere.cpp / EmitterCylinder.cpp inner loop).
void ring(double cx, double cz, double y, double r, double dtheta, std::vector<float>& out) {
    double theta = 0, theta_ap = 1;
    while (theta <= 2 * M_PI && theta_ap > 0) {
        push(out, cx + r * cos(theta), y, cz + r * sin(theta));
        theta += dtheta;
        theta_ap = theta;
    }
}

// EmitterSphere.cpp: layers from center.y up, then from center.y - rho down
void sphere(const psb_emitter& e, std::vector<float>& out) {
    const double cx = e.v[0], cy = e.v[1], cz = e.v[2];
    const float R = e.v[3], rho = e.particle_radius;
    auto layer = [&](double y) {
        double r = 0;
        while (r <= sqrt(R * R - y * y)) {
            ring(cx, cz, y, r, acos(r / sqrt(r * r + 2 * rho * rho)), out);
            r += rho;
        }
    };
    for (double y = cy; y < cy + R; y += rho) layer(y);
    for (double y = cy - rho; y >= cy - R; y -= rho) layer(y);
}

// EmitterCylinder.cpp
void cylinder(const psb_emitter& e, std::vector<float>& out) {
    const double cx = e.v[0], cy = e.v[1], cz = e.v[2];
    const double dy = e.v[4];
    const float rb = e.v[6], len = e.v[7], rho = e.particle_radius;
    const double p1y = cy + dy * (len / 2), p2y = cy - dy * (len / 2);
    for (double y = p2y; y < p1y; y += rho) {
        double r = 0;
        while (r <= rb) {
            ring(cx, cz, y, r, acos(r / sqrt(r * r + rho * rho)), out);
            r += rho;
        }
    }
}

// EmitterGirly.cpp: the grid [-3, 3]^3 at 0.02, x outer, z inner
void heart(std::vector<float>& out) {
    const double eps = 0.001, step = 0.02;
    for (double x = -3.0; x <= 3.0; x += step)
        for (double y = -3.0; y <= 3.0; y += step)
            for (double z = -3.0; z <= 3.0; z += step) {
                const double res = (double)powf((float)(x * x + 2 * y * y + z * z - 1), 3.f) - x * x * z * z * z -
                                   0 * y * y * z * z * z;
                if (res >= -eps && res <= eps) push(out, x, y, z);
            }
}

}  // namespace

extern "C" int psb_emitter_positions(const psb_emitter* e, int32_t emission, int64_t cap, float* out, int64_t* n) {
    if (!e || !n || cap < 0 || emission < 0) return PSB_EINVAL;
    std::vector<float> pos;
    switch (e->type) {
        case PSB_EMITTER_BOX: box(*e, pos); break;
        case PSB_EMITTER_SPHERE: sphere(*e, pos); break;
        case PSB_EMITTER_CYLINDER: cylinder(*e, pos); break;
        case PSB_EMITTER_HEART: heart(pos); break;
        case PSB_EMITTER_ELLIPSOID:
            if (e->count < 0) return PSB_EINVAL;
            pos.resize(3 * (size_t)e->count);
            for (int64_t i = 0; i < e->count; ++i)
                psb::emit::ellipsoid_point(e->v, e->seed, (uint32_t)emission, (uint64_t)i, &pos[3 * i]);
            break;
        case PSB_EMITTER_MESH: {
            if (e->count < 0 || e->n_faces < 0 || (e->n_faces > 0 && !e->data)) return PSB_EINVAL;
            const int64_t m = (int64_t)e->count * e->n_faces;
            pos.resize(3 * (size_t)m);
            for (int64_t i = 0; i < m; ++i)
                psb::emit::mesh_point(e->data + 9 * (i / e->count), e->seed, (uint32_t)emission, (uint64_t)i,
                                      &pos[3 * i]);
            break;
        }
        default:
            return PSB_EINVAL;
    }
    *n = (int64_t)(pos.size() / 3);
    if (out)
        for (int64_t i = 0; i < 3 * std::min<int64_t>(cap, *n); ++i) out[i] = pos[(size_t)i];
    return PSB_OK;
}
