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
#include <new>
#include <vector>

#include "psb.h"
#include "emitters.h"

namespace {

// The positions of one emission, bounded: a push beyond `limit` points
// stops the generator (TooMany) before the vector grows any further.
struct TooMany {};
struct Sink {
    std::vector<float>& v;
    size_t limit;
};

void push(Sink& out, double x, double y, double z) {
    if (out.v.size() / 3 >= out.limit) throw TooMany{};
    out.v.push_back((float)x);
    out.v.push_back((float)y);
    out.v.push_back((float)z);
}

// EmitterBox.cpp:29-47
void box(const psb_emitter& e, Sink& out) {
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
void ring(double cx, double cz, double y, double r, double dtheta, Sink& out) {
    double theta = 0, theta_ap = 1;
    while (theta <= 2 * M_PI && theta_ap > 0) {
        push(out, cx + r * cos(theta), y, cz + r * sin(theta));
        theta += dtheta;
        theta_ap = theta;
    }
}

// EmitterSphere.cpp: layers from center.y up, then from center.y - rho down
void sphere(const psb_emitter& e, Sink& out) {
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
void cylinder(const psb_emitter& e, Sink& out) {
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
void heart(Sink& out) {
    const double eps = 0.001, step = 0.02;
    for (double x = -3.0; x <= 3.0; x += step)
        for (double y = -3.0; y <= 3.0; y += step)
            for (double z = -3.0; z <= 3.0; z += step) {
                const double res = (double)powf((float)(x * x + 2 * y * y + z * z - 1), 3.f) - x * x * z * z * z -
                                   0 * y * y * z * z * z;
                if (res >= -eps && res <= eps) push(out, x, y, z);
            }
}

// The largest emission accepted: a context's particle count is an int32.
constexpr double kMaxPoints = 2147483647.0;

// True when adding `step` to any value of magnitude up to `mag` moves it by
// at least three quarters of a step (the step exceeds two ulps there), so a
// generator loop over that range advances.
bool advances_f(double mag, float step) {
    const float m = (float)std::fabs(mag);
    return std::isfinite(m) && step > 2 * (std::nextafter(m, INFINITY) - m);
}
bool advances_d(double mag, double step) {
    mag = std::fabs(mag);
    return std::isfinite(mag) && step > 2 * (std::nextafter(mag, INFINITY) - mag);
}
bool all_finite(const float* v, int k) {
    for (int i = 0; i < k; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

// Points on one ring of radius up to r with angular step atan(a / r), the
// ring loop's bound (dtheta only grows as the radius shrinks).
double ring_bound(double a, double r) { return 2 * M_PI / std::atan2(a, std::max(r, 0.0)) + 2; }

// An upper bound on the positions one emission of `e` produces, or -1 when
// the generator's loops would not end: a radius that is not positive, a value
// that is not finite, or a step below the resolution of the coordinates it
// advances. Every loop then advances by at least 3/4 of its step, which the
// per-axis counts (2 extent / step + 2) allow for.
double emission_bound(const psb_emitter& e) {
    const float rho = e.particle_radius;
    const bool rho_ok = rho > 0 && std::isfinite(rho);
    switch (e.type) {
        case PSB_EMITTER_BOX: {
            const float step = rho * 2;
            if (!rho_ok || !std::isfinite(step) || !all_finite(e.v, 9)) return -1;
            double b = 1;
            for (int a = 0; a < 3; ++a) {
                const double c = e.v[a], s = e.v[3 + a];
                if (!advances_f(std::fabs(c) + std::fabs(s), step)) return -1;
                b *= 2 * std::max(s, 0.0) / step + 2;
            }
            return b;
        }
        case PSB_EMITTER_SPHERE: {
            if (!rho_ok || !all_finite(e.v, 4)) return -1;
            const double R = std::max((double)e.v[3], 0.0);
            if (!advances_d(std::fabs((double)e.v[1]) + R + rho, rho)) return -1;
            return 2 * (2 * R / rho + 2) * (2 * R / rho + 2) * ring_bound(std::sqrt(2.0) * rho, R);
        }
        case PSB_EMITTER_CYLINDER: {
            if (!rho_ok || !all_finite(e.v, 8)) return -1;
            const double half = std::fabs((double)e.v[4] * ((double)e.v[7] / 2));
            const double rb = std::max((double)e.v[6], 0.0);
            if (!advances_d(std::fabs((double)e.v[1]) + half, rho) || !advances_d(rb + rho, rho)) return -1;
            return (4 * half / rho + 2) * (2 * rb / rho + 2) * ring_bound(rho, rb);
        }
        case PSB_EMITTER_HEART: return 301.0 * 301.0 * 301.0;
        case PSB_EMITTER_ELLIPSOID: return e.count < 0 ? -1 : (double)e.count;
        case PSB_EMITTER_MESH:
            if (e.count < 0 || e.n_faces < 0 || (e.n_faces > 0 && !e.data)) return -1;
            return (double)e.count * e.n_faces;
        default: return -1;
    }
}

}  // namespace

namespace psb {
namespace emit {

int generate(const psb_emitter& e, int32_t emission, int64_t limit, std::vector<float>& pos) {
    if (emission < 0 || limit < 0) return PSB_EINVAL;
    const double bound = emission_bound(e);
    if (!(bound >= 0 && bound <= kMaxPoints)) return PSB_EINVAL;
    pos.clear();
    if ((e.type == PSB_EMITTER_ELLIPSOID || e.type == PSB_EMITTER_MESH) && bound > (double)limit)
        return PSB_EOVERFLOW_NBR;     // the count is exact for the random emitters: nothing to generate
    Sink out{pos, (size_t)limit};
    try {
        switch (e.type) {
            case PSB_EMITTER_BOX: box(e, out); break;
            case PSB_EMITTER_SPHERE: sphere(e, out); break;
            case PSB_EMITTER_CYLINDER: cylinder(e, out); break;
            case PSB_EMITTER_HEART: heart(out); break;
            case PSB_EMITTER_ELLIPSOID:
                pos.resize(3 * (size_t)e.count);
                for (int64_t i = 0; i < e.count; ++i)
                    ellipsoid_point(e.v, e.seed, (uint32_t)emission, (uint64_t)i, &pos[3 * i]);
                break;
            case PSB_EMITTER_MESH: {
                const int64_t m = (int64_t)e.count * e.n_faces;
                pos.resize(3 * (size_t)m);
                for (int64_t i = 0; i < m; ++i)
                    mesh_point(e.data + 9 * (i / e.count), e.seed, (uint32_t)emission, (uint64_t)i, &pos[3 * i]);
                break;
            }
            default:
                return PSB_EINVAL;
        }
    } catch (const TooMany&) {
        pos.clear();
        return PSB_EOVERFLOW_NBR;
    } catch (const std::bad_alloc&) {
        pos.clear();
        return PSB_ENOMEM;
    }
    return PSB_OK;
}

}  // namespace emit
}  // namespace psb

extern "C" int psb_emitter_positions(const psb_emitter* e, int32_t emission, int64_t cap, float* out, int64_t* n) {
    if (!e || !n || cap < 0 || emission < 0) return PSB_EINVAL;
    std::vector<float> pos;
    const int rc = psb::emit::generate(*e, emission, (int64_t)kMaxPoints, pos);
    if (rc == PSB_EOVERFLOW_NBR) return PSB_EINVAL;
    if (rc != PSB_OK) return rc;
    *n = (int64_t)(pos.size() / 3);
    if (out)
        for (int64_t i = 0; i < 3 * std::min<int64_t>(cap, *n); ++i) out[i] = pos[(size_t)i];
    return PSB_OK;
}
