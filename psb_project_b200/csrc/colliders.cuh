// colliders.cuh -- the reference's collision objects (src/Kernel/Collision/*)
// as per-particle device functions: a finite plane, a sphere, a cylinder, a
// triangle mesh and height fields (linear, Gaussian, sums of cosines).
//
// Each object acts after the integrator on a particle's start position xo,
// its new position x and its new velocity v (for the SPH systems the
// leap-frog half-step velocity; SphSystem.cpp:323-328, CudaSystem.cpp:253-257)
// and, on a hit, moves x to the object's contact point and takes the normal
// part of v out, scaled by (1 + r) with the reference's restitution factor
// r = elast |x - x_contact| / (dt |v|).
//
// The formulas are the reference kernels' as they execute, including what
// the reference computes in float, and these behaviours of its code:
//  * plane (PlaneCollision_Kernel.cu:7-81): the in-quad test compares
//    x_a (1 - N_a) with the quad's extent scaled the same way, so it bounds
//    only the axes the normal does not lie along (with a negative normal
//    component it demands x_a on the quad's extent on that axis);
//    the contact is where the line from xo to x meets the plane.
//  * sphere (SphereCollision_Kernel.cu:7-91, SphereCollision.cu:9-16): its
//    launcher passes (elast, dt, container) where the kernel expects
//    (elast, container, dt), so the kernel's `container` is dt != 0 and its
//    dt is 1 or 0 (the caller's container flag). A sphere therefore always
//    keeps particles inside it; with container = false the restitution
//    divides by zero. Outside the container case the kernel only acts on a
//    particle exactly on the surface.
//  * cylinder (CylinderCollision_Kernel.cu:4-103): axis point
//    C = center + x * direction componentwise (its z uses direction.x),
//    a container of radius baseRadius - 0.04 and axial half length l/2,
//    restitution fixed at 0.3; the particle radius and container flag are
//    not read.
//  * mesh (MeshCollision_Kernel.cu:14-137): every face whose plane x lies
//    behind (d <= 0) is a candidate; the contact point is
//    xo + t (xo - x)/|xo - x| with t = ((A - x).N) / (dir.N) (measured from
//    x but applied at xo), kept if it projects into the triangle; a
//    particle on the plane or not moving (or d == -1) takes x itself with
//    no triangle test. The nearest candidate (last on ties) wins; the
//    restitution is 0 and N is used as stored.
//  * height fields (Linear/Gaussian/Periodic HeightFieldCollision_Kernel.cu):
//    inside the [min, max] footprint in x and z, y(x, z) = h(x, z) + min.y;
//    a particle at or below it is lifted to it, the normal from central
//    differences of h with step 0.01.
#pragma once
#include <cuda_runtime.h>

namespace psb {

enum : int { COLL_PLANE = 1, COLL_SPHERE = 2, COLL_CYLINDER = 3, COLL_MESH = 4, COLL_HEIGHT = 5 };
enum : int { HEIGHT_LINEAR = 1, HEIGHT_GAUSSIAN = 2, HEIGHT_COSINE = 3 };

// One object as the kernels read it. v[] by type:
//   plane: A, B, C, D (v[0..11]), N (v[12..14])
//   sphere: origin (v[0..2]), radius (v[3]); flag = the container argument
//   cylinder: center (v[0..2]), direction (v[3..5]), base radius (v[6]), length (v[7])
//   height: footprint min (v[0..2]) and max (v[3..5])
// Mesh faces: corners A, B, C and normal N of face i at fa/fb/fc/fn + i * stride.
// Height terms: 6 floats each, {kind, c0..c4}:
//   linear c0 x + c1 z; Gaussian c0 exp(-((x-c1)^2/(2 c3^2) + (z-c2)^2/(2 c4^2)));
//   cosine c0 cos(c1 (x cos c2 + z sin c2) + c3).
struct Collider {
    int type;
    int flag;
    float elast;
    int count;
    float v[16];
    const float* fa;
    const float* fb;
    const float* fc;
    const float* fn;
    int stride;
    const float* terms;
};

namespace coll {

template <typename T>
struct V3 {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T>
__device__ __forceinline__ V3<T> sub(V3<T> a, V3<T> b) { return mk<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T>
__device__ __forceinline__ T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
__device__ __forceinline__ T len(V3<T> a) { return sqrt(dot(a, a)); }
// componentwise division (double3.h normalize)
template <typename T>
__device__ __forceinline__ V3<T> divided(V3<T> a, T l) { return mk<T>(a.x / l, a.y / l, a.z / l); }
// multiplication by the reciprocal (double3.h operator/)
template <typename T>
__device__ __forceinline__ V3<T> over(V3<T> a, T l) {
    const T r = (T)1.0f / l;
    return mk<T>(a.x * r, a.y * r, a.z * r);
}
__device__ __forceinline__ V3<float> f3v(const float* p) { return mk<float>(p[0], p[1], p[2]); }
template <typename T>
__device__ __forceinline__ V3<T> widen(V3<float> a) { return mk<T>((T)a.x, (T)a.y, (T)a.z); }
template <typename T>
__device__ __forceinline__ V3<float> narrow(V3<T> a) { return mk<float>((float)a.x, (float)a.y, (float)a.z); }
// float square of a value the reference passes through powf(., 2)
__device__ __forceinline__ float fsq(float a) { return a * a; }

// v -= (1 + r) (v.n) n; r is float in the reference kernels
template <typename T>
__device__ __forceinline__ void reflect(V3<T>& v, V3<T> n, float r) {
    const T k = (T)(1.f + r) * dot(v, n);
    v = mk<T>(v.x - k * n.x, v.y - k * n.y, v.z - k * n.z);
}

// r = elast |x - xc| / (dt |v|) when |v| > 0 and elast > 0
template <typename T>
__device__ __forceinline__ float restitution(float elast, float dt, V3<T> x, V3<T> xc, V3<T> v) {
    const T lv = len(v);
    if (lv > 0 && elast > 0) return (float)((T)elast * len(sub(x, xc)) / ((T)dt * lv));
    return 0.f;
}

// ---- plane (PlaneCollision_Kernel.cu) -------------------------------------
template <typename T>
__device__ bool plane(const Collider& o, float dt, V3<T> xo, V3<T>& x, V3<T>& v) {
    const float* q = o.v;
    const V3<float> N = f3v(q + 12), A = f3v(q);
    float lo[3] = {100000.f, 100000.f, 100000.f}, hi[3] = {-100000.f, -100000.f, -100000.f};
    for (int c = 0; c < 4; ++c)
        for (int a = 0; a < 3; ++a) {
            const float e = q[3 * c + a];
            if (lo[a] >= e) lo[a] = e;
            if (hi[a] <= e) hi[a] = e;
        }
    const T xs[3] = {x.x, x.y, x.z};
    const float ns[3] = {N.x, N.y, N.z};
    for (int a = 0; a < 3; ++a) {
        const float s = 1.f - ns[a];
        const T xa = xs[a] * (T)s;
        if (!(xa <= (T)(hi[a] * s) && xa >= (T)(lo[a] * s))) return false;
    }
    const V3<float> p1 = narrow(sub(x, widen<T>(A)));
    if (!(dot(p1, N) <= 0.f)) return false;
    const float ao_n = dot(narrow(sub(widen<T>(A), xo)), N);
    V3<float> dir = narrow(sub(x, xo));
    const float dn = sqrtf(dot(dir, dir));
    if (!(dn > 0.f)) return false;   // no motion: the reference divides by zero
    dir = mk<float>(dir.x / dn, dir.y / dn, dir.z / dn);
    const float t = ao_n / dot(dir, N);
    const V3<T> xc = mk<T>(xo.x + (T)(t * dir.x), xo.y + (T)(t * dir.y), xo.z + (T)(t * dir.z));
    const float r = restitution<T>(o.elast, dt, x, xc, v);
    const V3<T> n = divided(widen<T>(N), len(widen<T>(N)));
    x = xc;
    reflect(v, n, r);
    return true;
}

// ---- sphere (SphereCollision_Kernel.cu through SphereCollision.cu's launch) --
template <typename T>
__device__ bool sphere(const Collider& o, float dt, V3<T> x_unused, V3<T>& x, V3<T>& v) {
    (void)x_unused;
    const bool inside = dt != 0.f;               // the kernel's `container`
    const float dt_k = o.flag ? 1.f : 0.f;       // the kernel's `dt`
    const V3<T> c = widen<T>(f3v(o.v));
    const T R = (T)o.v[3];
    const V3<T> op = sub(x, c);
    const T d = len(op);
    V3<T> xc, n;
    if (inside && d >= R) {
        if (d == R) {
            xc = x;
            n = over(mk<T>(-op.x, -op.y, -op.z), d);
        } else {
            const V3<T> u = over(op, d);
            xc = mk<T>(c.x + u.x * R, c.y + u.y * R, c.z + u.z * R);
            const V3<T> w = sub(c, xc);
            n = over(w, len(w));
        }
    } else if (!inside && d == R) {
        xc = x;
        n = over(mk<T>(-op.x, -op.y, -op.z), d);
    } else {
        return false;
    }
    const float r = restitution<T>(o.elast, dt_k, x, xc, v);
    n = divided(n, len(n));
    x = xc;
    reflect(v, n, r);
    return true;
}

// ---- cylinder (CylinderCollision_Kernel.cu) ---------------------------------
template <typename T>
__device__ bool cylinder(const Collider& o, float dt, V3<T> x_unused, V3<T>& x, V3<T>& v) {
    (void)x_unused;
    const V3<float> ce = f3v(o.v), di = f3v(o.v + 3);
    const float rb = o.v[6], l = o.v[7];
    const V3<T> p1 = mk<T>((T)(ce.x + di.x * (l / 2)), (T)(ce.y + di.y * (l / 2)), (T)(ce.z + di.z * (l / 2)));
    const V3<T> p2 = mk<T>((T)(ce.x - di.x * (l / 2)), (T)(ce.y - di.y * (l / 2)), (T)(ce.z - di.z * (l / 2)));
    const V3<T> C = mk<T>((T)ce.x + x.x * (T)di.x, (T)ce.y + x.y * (T)di.y, (T)ce.z + x.z * (T)di.x);
    const T margin = (T)rb - (T)0.04;
    auto fdist = [](V3<T> a, V3<T> b) {
        return (T)sqrtf(fsq((float)(a.x - b.x)) + fsq((float)(a.y - b.y)) + fsq((float)(a.z - b.z)));
    };
    const T dist = fdist(widen<T>(ce), C);
    V3<T> xc = x, n;
    const float dl = sqrtf(fsq(di.x) + fsq(di.y) + fsq(di.z));
    if (dist >= (T)(l / 2)) {
        const T d1 = fdist(p1, C), d2 = fdist(p2, C);
        const V3<T> w = sub(C, x);
        const T lw = len(w);
        const bool low = d1 > d2;            // nearer the P2 end
        const T s = low ? (T)1 : (T)-1;
        const V3<T> u = mk<T>(s * w.x / lw, s * w.y / lw, s * w.z / lw);
        const V3<T> pe = low ? p2 : p1;
        if (di.x != 0.f) xc.x = pe.x;
        if (di.y != 0.f) xc.y = pe.y;
        if (di.z != 0.f) xc.z = pe.z;
        if (lw >= (T)rb) {
            // P2 side: C - margin u with u toward the axis; P1 side: C + margin u with u away from it
            if (di.x == 0.f) xc.x = C.x - s * margin * u.x;
            if (di.y == 0.f) xc.y = C.y - s * margin * u.y;
            if (di.z == 0.f) xc.z = C.z - s * margin * u.z;
        }
        const float sn = low ? 1.f : -1.f;
        n = mk<T>((T)(sn * di.x) / (T)dl, (T)(sn * di.y) / (T)dl, (T)(sn * di.z) / (T)dl);
    } else {
        if (!(fdist(C, x) >= (T)rb)) return false;
        const V3<T> w = sub(C, x);
        const T lw = len(w);
        const V3<T> u = mk<T>(-w.x / lw, -w.y / lw, -w.z / lw);
        xc = mk<T>(C.x + margin * u.x * (T)(1.f - di.x), C.y + margin * u.y * (T)(1.f - di.y),
                   C.z + margin * u.z * (T)(1.f - di.z));
        n = u;
    }
    float r = 0.f;
    const T lv = len(v);
    if (lv > 0 && dt > 0.f) r = (float)((T)0.3f * len(sub(x, xc)) / ((T)dt * lv));
    x = xc;
    reflect(v, n, r);
    return true;
}

// ---- triangle mesh (MeshCollision_Kernel.cu) --------------------------------
__device__ __forceinline__ bool in_triangle(V3<float> A, V3<float> B, V3<float> C, V3<float> P) {
    const V3<float> u = sub(B, A), w = sub(C, A), p = sub(P, A);
    const float uu = dot(u, u), uw = dot(u, w), ww = dot(w, w), pu = dot(p, u), pw = dot(p, w);
    const float D = uw * uw - uu * ww;
    const float s = (uw * pw - ww * pu) / D;
    if (s < 0.f || s > 1.f) return false;
    const float t = (uw * pu - uu * pw) / D;
    if (t < 0.f || (s + t) > 1.f) return false;
    return true;
}

template <typename T>
__device__ bool mesh(const Collider& o, float dt, V3<T> xo, V3<T>& x, V3<T>& v) {
    (void)dt;
    T best = (T)10000000;
    bool found = false;
    V3<T> xb = x;
    V3<float> nb = mk<float>(0.f, 0.f, 0.f);
    for (int f = 0; f < o.count; ++f) {
        const long long at = (long long)f * o.stride;
        const V3<float> A = f3v(o.fa + at), N = f3v(o.fn + at);
        const T d1 = dot(sub(x, widen<T>(A)), widen<T>(N));
        if (!(d1 <= 0)) continue;
        const V3<T> dir0 = sub(xo, x);
        const T dn = len(dir0);
        V3<T> xc;
        if (d1 == 0 || dn <= 0 || d1 == (T)-1) {
            xc = x;
        } else {
            const T ao_n = dot(sub(widen<T>(A), x), widen<T>(N));
            const V3<T> dir = divided(dir0, dn);
            const T t = ao_n / dot(dir, widen<T>(N));
            xc = mk<T>(xo.x + t * dir.x, xo.y + t * dir.y, xo.z + t * dir.z);
            if (!in_triangle(A, f3v(o.fb + at), f3v(o.fc + at), narrow(xc))) continue;
        }
        const T dist =
            (T)sqrtf(fsq((float)(x.x - xc.x)) + fsq((float)(x.y - xc.y)) + fsq((float)(x.z - xc.z)));
        if (dist <= best) {
            best = dist;
            xb = xc;
            nb = N;
            found = true;
        }
    }
    if (!found) return false;
    x = xb;
    reflect(v, widen<T>(nb), 0.f);
    return true;
}

// ---- height fields ------------------------------------------------------------
// Footprint test, lift and reflection shared by every height function h.
template <typename T, typename H>
__device__ bool height(const Collider& o, float dt, V3<T>& x, V3<T>& v, H h) {
    const float* q = o.v;
    if (!(x.x >= (T)q[0] && x.z >= (T)q[2] && x.x <= (T)q[3] && x.z <= (T)q[5])) return false;
    const T y = h(x.x, x.z) + (T)q[1];
    if (!(y >= x.y)) return false;
    const V3<T> xc = mk<T>(x.x, y, x.z);
    const float r = restitution<T>(o.elast, dt, x, xc, v);
    const T d = (T)0.01;
    const T dpx = (h(xc.x + d, xc.z) - h(xc.x - d, xc.z)) / (2 * d);
    const T dpz = (h(xc.x, xc.z + d) - h(xc.x, xc.z - d)) / (2 * d);
    const T nn = sqrt(dpx * dpx + (T)1 + dpz * dpz);
    V3<T> n = mk<T>(-dpx / nn, (T)1 / nn, -dpz / nn);
    n = divided(n, len(n));
    x = xc;
    reflect(v, n, r);
    return true;
}

// The terms of a native height object, summed in order (float).
struct TermSum {
    const float* t;
    int count;
    __device__ float operator()(float x, float z) const {
        float y = 0.f;
        for (int i = 0; i < count; ++i) {
            const float* c = t + 6 * i;
            const int kind = (int)c[0];
            if (kind == HEIGHT_LINEAR) {
                y += c[1] * x + c[2] * z;
            } else if (kind == HEIGHT_GAUSSIAN) {
                y += c[1] * expf(-(fsq(x - c[2]) / (2 * c[4] * c[4]) + fsq(z - c[3]) / (2 * c[5] * c[5])));
            } else {
                y += c[1] * cosf(c[2] * (x * cosf(c[3]) + z * sinf(c[3])) + c[4]);
            }
        }
        return y;
    }
};

// Every object of the list in order (native path, FP32 state).
__device__ __forceinline__ void apply_colliders(const Collider* objs, int n, float dt, V3<float> xo, V3<float>& x,
                                                V3<float>& v) {
    for (int k = 0; k < n; ++k) {
        const Collider& o = objs[k];
        switch (o.type) {
            case COLL_PLANE: plane<float>(o, dt, xo, x, v); break;
            case COLL_SPHERE: sphere<float>(o, dt, xo, x, v); break;
            case COLL_CYLINDER: cylinder<float>(o, dt, xo, x, v); break;
            case COLL_MESH: mesh<float>(o, dt, xo, x, v); break;
            case COLL_HEIGHT: height<float>(o, dt, x, v, TermSum{o.terms, o.count}); break;
            default: break;
        }
    }
}

}  // namespace coll
}  // namespace psb
