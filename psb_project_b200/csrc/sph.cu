// sph.cu -- SPH density, forces and the PCISPH predictor-corrector sweeps.
//
// One thread per cell-sorted particle, walking its neighbour list (slot-
// major, so a warp's list reads are coalesced). Sums are per-particle and
// atomic-free, in the list's fixed order; densities use Kahan-compensated
// FP32 sums. All kernel constants are pre-scaled (q = r^2/h^2, u = r/h) so
// FP32 never sees h^9.
//
// Formulas and their reference sources (paths inside the reference tree):
//   density  rho_i = m 315/(64 pi h^9) sum (h^2-r^2)^3
//            SphKernel.cu:9-27, PciSphSystem_Kernel.cu:70-85
//   pressure force density -rho_i sum m (p_i/rho_i^2 + p_j/rho_j^2) gradW,
//            gradW = -45/(pi h^6) (h-r)^2 r^     SphKernel.cu:53-61, PciSphSystem_Kernel.cu:88-114
//   viscosity sum mu (v_j-v_i) m/rho_j 45 (h-r)/(pi h^6)
//            SphKernel.cu:63-66, PciSphSystem_Kernel.cu:141-146
//   surface tension and normals (reference profile only)
//            SphKernel.cu:68-88, PciSphSystem_Kernel.cu:148-166
//   PCISPH pressure increment (rho*-rho0)/(beta(|sum gradW|^2 + sum|gradW|^2)),
//            compressed particles only     PciSphSystem_Kernel.cu:36-67
//            (config profile: Solenthaler & Pajarola's prototype factor for every
//            particle, p clamped at 0; the per-particle form diverges when
//            iterated to an eta, see the config notes in the oracle)
//   leap-frog v+ += a dt, x += v+ dt; v = (v- + v+)/2
//            SphKernel.cu:95-135
//   box walls: projection + reflection     BoxCollision_Kernel.cu:7-34
// The reference's predict/restore passes (PciSphSystem.cu:30-61) become a
// predictor that writes x*, v* to separate buffers and leaves the state
// alone; the final leap-frog is the last prediction committed.
#include <algorithm>
#include <cooperative_groups.h>

#include "psb_internal.cuh"
#include "colliders.cuh"

namespace cg = cooperative_groups;

namespace psb {

namespace {

// The sums that several kernels compute for the same pair (the corrector's
// passes in their own kernels and in the persistent one, the density at x in
// its own sweep and inside the neighbour build) round the same way in every
// kernel: wherever a product feeds a sum, the operation is written out --
// __fmaf_rn where the product is fused, __fmul_rn/__fadd_rn/__fsub_rn (never
// contracted) where it is not. Plain * and + remain only where no fused
// multiply-add can form (products of products, a sum feeding a product), so
// the results do not depend on where the compiler would fuse.
struct Kahan {
    float s = 0.f, c = 0.f;     // sum and (negated) lost low part: true sum ~ s - c
    __device__ __forceinline__ void add(float x) {
        const float y = __fsub_rn(x, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    // adds a * b with the product rounded only inside the sum (one FMA)
    __device__ __forceinline__ void add_prod(float a, float b) {
        const float y = __fmaf_rn(a, b, -c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
};

// Adds a pair's (1 - q)^3, q = r2 / h^2 < 1, as (1 - q)^2 times (1 - q).
__device__ __forceinline__ void add_poly6(Kahan& acc, float q) {
    const float w = __fsub_rn(1.f, q);
    acc.add_prod(__fmul_rn(w, w), w);
}

// 1 - r/h of a pair, from r2 and its reciprocal square root
__device__ __forceinline__ float spiky_om(const Params& P, float r2, float rinv) {
    return __fmaf_rn(-(r2 * rinv), P.inv_h, 1.f);
}

// rho - rho0 = k_rho (s - c) - rho0 with the product's low part kept by the
// FMA: the deviation, from which every pressure is computed, keeps its full
// relative precision instead of the ~6e-5 absolute step of an FP32 density.
__device__ __forceinline__ float density_deviation(const Params& P, const Kahan& a) {
    return __fsub_rn(__fmaf_rn(P.k_rho, a.s, -P.rho0), __fmul_rn(P.k_rho, a.c));
}

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }

// The box faces that bound particle t (slot t): the scene's own (kernel
// parameters, read where used) or, in a batch, its scene's table entry.
template <bool BATCH> struct Faces;
template <> struct Faces<false> {
    const Params& P;
    __device__ __forceinline__ float x0() const { return P.bx0; }
    __device__ __forceinline__ float y0() const { return P.by0; }
    __device__ __forceinline__ float z0() const { return P.bz0; }
    __device__ __forceinline__ float x1() const { return P.bx1; }
    __device__ __forceinline__ float y1() const { return P.by1; }
    __device__ __forceinline__ float z1() const { return P.bz1; }
};
template <> struct Faces<true> {
    const SceneGeom* G;
    __device__ __forceinline__ float x0() const { return G->bx0; }
    __device__ __forceinline__ float y0() const { return G->by0; }
    __device__ __forceinline__ float z0() const { return G->bz0; }
    __device__ __forceinline__ float x1() const { return G->bx1; }
    __device__ __forceinline__ float y1() const { return G->by1; }
    __device__ __forceinline__ float z1() const { return G->bz1; }
};
template <bool BATCH>
__device__ __forceinline__ Faces<BATCH> faces_of(const Params& P, int t);
template <>
__device__ __forceinline__ Faces<false> faces_of<false>(const Params& P, int) { return Faces<false>{P}; }
template <>
__device__ __forceinline__ Faces<true> faces_of<true>(const Params& P, int t) {
    return Faces<true>{P.scenes + P.slot_scene[t]};
}

// Penalty walls (config profile): a = K*depth - C*v along each axis on which
// x lies outside the box (a state uploaded outside it; the projection below
// keeps stepped particles inside).
template <bool REF, bool BATCH = false>
__device__ __forceinline__ float3 wall_accel(const Params& P, int t, float4 x, float4 v) {
    float3 a = make_float3(0.f, 0.f, 0.f);
    if (REF) return a;
    const auto F = faces_of<BATCH>(P, t);
    // K * depth - C * v, depth > 0 on the outside
    auto push = [&](float depth, float vel) {
        return __fsub_rn(__fmul_rn(P.wall_k, depth), __fmul_rn(P.wall_c, vel));
    };
    if (x.x < F.x0()) a.x = __fadd_rn(a.x, push(__fsub_rn(F.x0(), x.x), v.x));
    if (x.x > F.x1()) a.x = __fadd_rn(a.x, push(-__fsub_rn(x.x, F.x1()), v.x));
    if (x.y < F.y0()) a.y = __fadd_rn(a.y, push(__fsub_rn(F.y0(), x.y), v.y));
    if (x.y > F.y1()) a.y = __fadd_rn(a.y, push(-__fsub_rn(x.y, F.y1()), v.y));
    if (x.z < F.z0()) a.z = __fadd_rn(a.z, push(__fsub_rn(F.z0(), x.z), v.z));
    if (x.z > F.z1()) a.z = __fadd_rn(a.z, push(-__fsub_rn(x.z, F.z1()), v.z));
    return a;
}

// Config-profile walls: mirror ghost particles (Libersky et al. 1993;
// Colagrossi & Landrini 2003). Every box face within h of particle i
// reflects i's neighbours (self included); for each non-empty set S of such
// faces, the ghost of j is j reflected across every face in S, provided j is
// itself within h of each. A ghost can only lie within h of i if j does, so
// the neighbour list yields all of them. Ghosts carry j's pressure continued
// hydrostatically across the faces, p_j + rho0 (-g . n) 2 d_j, so a resting
// column is held by its bottom layer as by any interior layer.
// The faces near a particle, packed in one word: bits 0-1 hold their count
// n (at most one face per axis), and face k takes 3 bits at 2 + 3k: its axis
// (2 bits) and whether it is the lower face (inward normal +1).
__device__ __forceinline__ float comp(float4 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ float gcomp(const Params& P, int a) { return a == 0 ? P.gx : (a == 1 ? P.gy : P.gz); }

template <class F_>
__device__ __forceinline__ unsigned near_walls(const Params& P, const F_& F, float4 x) {
    unsigned w = 0u, n = 0u;
    auto push = [&](unsigned axis, unsigned lower) { w |= (axis | (lower << 2)) << (2u + 3u * n); ++n; };
    if (x.x - F.x0() < P.hf) push(0u, 1u);
    else if (F.x1() - x.x < P.hf) push(0u, 0u);
    if (x.y - F.y0() < P.hf) push(1u, 1u);
    else if (F.y1() - x.y < P.hf) push(1u, 0u);
    if (x.z - F.z0() < P.hf) push(2u, 1u);
    else if (F.z1() - x.z < P.hf) push(2u, 0u);
    return w | n;
}

// Reflects the offset across face k of w: with d = nrm (x - plane) the
// distances on the box side, component a of r becomes nrm (d_i + d_j), both
// clamped at 0 so that a particle pushed through the face still sees its
// ghosts on the wall side (unclamped, its own ghost would push it further
// out). False if x_j is h or more inside.
template <class F_>
__device__ __forceinline__ bool reflect(const Params& P, const F_& F, unsigned w, int k, float4 xi, float4 xj,
                                        float3& r, float& dp) {
    const unsigned f = (w >> (2 + 3 * k)) & 7u;
    const int a = (int)(f & 3u);
    const bool lower = (f >> 2) != 0u;
    const float plane = lower ? (a == 0 ? F.x0() : (a == 1 ? F.y0() : F.z0()))
                              : (a == 0 ? F.x1() : (a == 1 ? F.y1() : F.z1()));
    const float nrm = lower ? 1.f : -1.f;
    const float dj = fmaxf(__fmul_rn(nrm, __fsub_rn(comp(xj, a), plane)), 0.f);
    if (dj >= P.hf) return false;
    const float di = fmaxf(__fmul_rn(nrm, __fsub_rn(comp(xi, a), plane)), 0.f);
    const float v = __fmul_rn(nrm, __fadd_rn(di, dj));
    if (a == 0) r.x = v; else if (a == 1) r.y = v; else r.z = v;
    dp = __fmaf_rn(__fmul_rn(__fmul_rn(P.rho0, __fmul_rn(-gcomp(P, a), nrm)), 2.f), dj, dp);
    return true;
}

// x_i minus the ghost of x_j across the faces in `mask`; false if a face of
// the set is h or more from x_j. dp: the ghost's hydrostatic pressure offset.
template <class F_>
__device__ __forceinline__ bool ghost_delta(const Params& P, const F_& F, unsigned w, int mask, float4 xi,
                                            float4 xj, float3& r, float& dp) {
    r = make_float3(__fsub_rn(xi.x, xj.x), __fsub_rn(xi.y, xj.y), __fsub_rn(xi.z, xj.z));
    dp = 0.f;
    if ((mask & 1) && !reflect(P, F, w, 0, xi, xj, r, dp)) return false;
    if ((mask & 2) && !reflect(P, F, w, 1, xi, xj, r, dp)) return false;
    if ((mask & 4) && !reflect(P, F, w, 2, xi, xj, r, dp)) return false;
    return true;
}

// The ghosts of neighbour x_j (one per non-empty subset of the near faces).
// Density: adds (1-q)^3 of each ghost within h.
template <class F_>
__device__ __forceinline__ void ghost_density_pair(const Params& P, const F_& F, unsigned w, float4 xi, float4 xj,
                                                   Kahan& acc) {
    const int nm = 1 << (w & 3u);
    for (int mask = 1; mask < nm; ++mask) {
        float3 r;
        float dp;
        if (!ghost_delta(P, F, w, mask, xi, xj, r, dp)) continue;
        const float q = __fmul_rn(dist2(r.x, r.y, r.z), P.inv_h2);
        if (q >= 1.f) continue;
        add_poly6(acc, q);
    }
}

// Pressure: adds (pV_i + pV_ghost) (1-u)^2 x^ of each ghost within h, the
// ghost carrying p_j continued hydrostatically across its faces.
template <class F_>
__device__ __forceinline__ void ghost_pressure_pair(const Params& P, const F_& F, unsigned w, float4 xi, float4 xj,
                                                    float pVi, float pj, float3& ap) {
    const float ir0 = 1.f / __fmul_rn(P.rho0, P.rho0);
    const int nm = 1 << (w & 3u);
    for (int mask = 1; mask < nm; ++mask) {
        float3 r;
        float dp;
        if (!ghost_delta(P, F, w, mask, xi, xj, r, dp)) continue;
        const float r2 = dist2(r.x, r.y, r.z);
        if (!(r2 > 0.f) || __fmul_rn(r2, P.inv_h2) >= 1.f) continue;
        const float rinv = rsqrtf(r2);
        const float om = spiky_om(P, r2, rinv);
        const float sc = __fmul_rn(__fmul_rn(__fmul_rn(__fmaf_rn(__fadd_rn(pj, dp), ir0, pVi), om), om), rinv);
        ap.x = __fmaf_rn(sc, r.x, ap.x); ap.y = __fmaf_rn(sc, r.y, ap.y); ap.z = __fmaf_rn(sc, r.z, ap.z);
    }
}

// Ghost terms of particle t, in a second walk of its list that only
// particles within h of a face take (the walls are evaluated at xi). Kept
// out of the main walk: a per-neighbour wall test there slows every
// particle more than the separate walk costs the few near the faces.
// The positions (ghost_density) and pressures (ghost_pressure) may be ones
// that the persistent corrector rewrites between its passes, so they are
// not declared __restrict__ here: a kernel whose own arguments are
// restrict-qualified read-only arrays still gets read-only-cache loads.
template <bool BATCH = false>
__device__ __forceinline__ void ghost_density(const Params& P, int t, float4 xi, const float4* pos,
                                              const int* __restrict__ list, int cnt, Kahan& acc) {
    const auto F = faces_of<BATCH>(P, t);
    const unsigned wall = near_walls(P, F, xi);
    if (!(wall & 3u)) return;
    for_each_nbr(list, P.n, t, cnt, [&](const int j) { ghost_density_pair(P, F, wall, xi, pos[j], acc); });
}

template <bool BATCH = false>
__device__ __forceinline__ void ghost_pressure(const Params& P, int t, float4 xi, float pVi,
                                               const float4* __restrict__ pos, const float* pj_of,
                                               int pj_stride, const int* __restrict__ list, int cnt, float3& ap) {
    const auto F = faces_of<BATCH>(P, t);
    const unsigned wall = near_walls(P, F, xi);
    if (!(wall & 3u)) return;
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        ghost_pressure_pair(P, F, wall, xi, pos[j], pVi, pj_of[(size_t)j * pj_stride], ap);
    });
}

// Boundary particles (config profile; boundary.cu): density psi_b W_ib, as
// (psi_b / m) (1 - q)^3 inside the k_rho-scaled sum, and the mirrored
// pressure term psi_b pV_i gradW_ib, as (psi_b / m) pV_i (1-u)^2 x^ inside
// the k_grad-scaled sum. The positions are the step's start positions of
// a static solid; x_i is the particle's current (or predicted) position.
// bx: the boundary positions the density sees (P.bnd at the step's start
// positions; in the corrector, P.bnd_pred where the boundary moves with it).
__device__ __forceinline__ void boundary_density(const Params& P, int t, float4 xi, Kahan& acc,
                                                 const float4* __restrict__ bx) {
    if (!P.bnd_count) return;
    const int cnt = min(P.bnd_count[t], P.bnd_cap);
    for_each_nbr(P.bnd_list, P.n, t, cnt, [&](const int b) {
        const float4 xb = bx[b];
        const float dx = __fsub_rn(xi.x, xb.x), dy = __fsub_rn(xi.y, xb.y), dz = __fsub_rn(xi.z, xb.z);
        const float q = __fmul_rn(dist2(dx, dy, dz), P.inv_h2);
        if (q >= 1.f) return;
        const float w = __fsub_rn(1.f, q);
        acc.add_prod(xb.w, __fmul_rn(__fmul_rn(w, w), w));
    });
}

__device__ __forceinline__ void boundary_pressure(const Params& P, int t, float4 xi, float pVi, float3& ap) {
    if (!P.bnd_count) return;
    const int cnt = min(P.bnd_count[t], P.bnd_cap);
    for_each_nbr(P.bnd_list, P.n, t, cnt, [&](const int b) {
        const float4 xb = P.bnd[b];
        const float dx = __fsub_rn(xi.x, xb.x), dy = __fsub_rn(xi.y, xb.y), dz = __fsub_rn(xi.z, xb.z);
        const float r2 = dist2(dx, dy, dz);
        if (!(r2 > 0.f) || __fmul_rn(r2, P.inv_h2) >= 1.f) return;
        const float rinv = rsqrtf(r2);
        const float om = spiky_om(P, r2, rinv);
        const float sc = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(xb.w, pVi), om), om), rinv);
        ap.x = __fmaf_rn(sc, dx, ap.x); ap.y = __fmaf_rn(sc, dy, ap.y); ap.z = __fmaf_rn(sc, dz, ap.z);
    });
}

// collisionBox (BoxCollision_Kernel.cu:7-34) with restitution 0: clamp into
// [Min+r, Max-r] (upper bounds tested first, lower bounds win), then remove
// the velocity component along the normalised sum of wall normals. PCISPH
// in both profiles: in the config profile it keeps every particle at least r
// from each face, where its own ghost still pushes back (a particle on or
// behind a face meets its ghost at distance 0, which exerts no force, and
// its density error could not be corrected). Config WCSPH keeps the penalty
// walls its scene states.
template <bool BATCH = false>
__device__ __forceinline__ void box_project(const Params& P, int t, float3& x, float3& v) {
    float wlo_x = P.wlo_x, wlo_y = P.wlo_y, wlo_z = P.wlo_z, whi_x = P.whi_x, whi_y = P.whi_y, whi_z = P.whi_z;
    if (BATCH) {
        const SceneGeom* G = P.scenes + P.slot_scene[t];
        wlo_x = G->wlo_x; wlo_y = G->wlo_y; wlo_z = G->wlo_z; whi_x = G->whi_x; whi_y = G->whi_y; whi_z = G->whi_z;
    }
    float3 pI = x, nI = make_float3(0.f, 0.f, 0.f);
    if (x.x >= whi_x) { pI.x = whi_x; nI.x = -1.f; }
    if (x.y >= whi_y) { pI.y = whi_y; nI.y = -1.f; }
    if (x.z >= whi_z) { pI.z = whi_z; nI.z = -1.f; }
    if (x.x <= wlo_x) { pI.x = wlo_x; nI.x = 1.f; }
    if (x.y <= wlo_y) { pI.y = wlo_y; nI.y = 1.f; }
    if (x.z <= wlo_z) { pI.z = wlo_z; nI.z = 1.f; }
    const float l2 = nI.x * nI.x + nI.y * nI.y + nI.z * nI.z;
    if (l2 > 0.f) {
        const float il = rsqrtf(l2);
        nI.x *= il; nI.y *= il; nI.z *= il;
        const float vd = v.x * nI.x + v.y * nI.y + v.z * nI.z;
        x = pI;
        v.x -= vd * nI.x; v.y -= vd * nI.y; v.z -= vd * nI.z;
    }
}

// ---- density at the step's start positions ---------------------------------
// WCSPH: also the equation of state (reference: p = k (rho - rho0),
// SphKernel.cu:25; config: Tait, p = k rho0/7 ((rho/rho0)^7 - 1), written as
// k rho0/7 d (1 + x + ... + x^6) with x = 1 + d to avoid cancellation).
// PCISPH: keeps the carried pressure (warm start) or zeroes it.
// NF (config PCISPH, learned warm start or data collection): the same
// neighbour walk also sums the velocity divergence and density gradient and
// writes the MLP's first NF inputs (6 or 7; feats, stride 8, the rest 0):
//   f0 neighbour count / 32
//   f1 advected density deviation (rho - dt rho div v - rho0)/rho0 * 100
//   f2 div v * dt * 100, div v = -(k_grad/rho0) sum (1-u)^2 (v_j - v_i).x^
//   f3 previous-step pressure / p_scale
//   f4 distance to the nearest box face / h, capped at 1
//   f5 k_grad |sum (1-u)^2 x^| h / rho0 (density-gradient magnitude)
//   f6 sum W_ij p_j / sum W_ij / p_scale over the list, self included: the
//      carried pressure smoothed with the poly6 weights
// The sums of the density pass at x for one particle, pair by pair in list
// order; shared by the density sweep and by the neighbour build that
// computes the density as it accepts each neighbour, so that both give the
// same bits.
template <bool REF, int NF>
struct DensityX {
    static constexpr bool FEAT = NF > 0, SMOOTH_P = NF > 6;
    Kahan acc;
    float div = 0.f, wp = 0.f, ws = 0.f;
    float3 gr = make_float3(0.f, 0.f, 0.f);
    float4 vi = make_float4(0.f, 0.f, 0.f, 0.f);

    __device__ __forceinline__ void begin(const float4* __restrict__ vel, int t) {
        if (FEAT) vi = vel[t];
    }
    // neighbour j at xj (r2 = dist2 of xi - xj); rp[j].y is the carried
    // pressure, which the pass writes back unchanged
    __device__ __forceinline__ void pair(const Params& P, float4 xi, float4 xj, int j, const float4* __restrict__ vel,
                                         const float2* __restrict__ rp) {
        // the pair's other gathers issue with its position, ahead of the tests
        const float4 vj = FEAT ? vel[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float pj = SMOOTH_P ? rp[j].y : 0.f;
        const float dx = __fsub_rn(xi.x, xj.x), dy = __fsub_rn(xi.y, xj.y), dz = __fsub_rn(xi.z, xj.z);
        const float r2 = dist2(dx, dy, dz);
        const float q = __fmul_rn(r2, P.inv_h2);
        if (!REF && q >= 1.f) return;
        const float w = __fsub_rn(1.f, q);
        const float w2 = __fmul_rn(w, w);
        const float w3 = __fmul_rn(w2, w);
        acc.add_prod(w2, w);
        if (SMOOTH_P) {
            wp = __fmaf_rn(w3, pj, wp);
            ws = __fadd_rn(ws, w3);
        }
        if (FEAT && r2 > 0.f) {
            const float rinv = rsqrtf(r2);
            const float om = spiky_om(P, r2, rinv);
            const float s = __fmul_rn(__fmul_rn(om, om), rinv);           // (1-u)^2 / r
            gr.x = __fmaf_rn(s, dx, gr.x); gr.y = __fmaf_rn(s, dy, gr.y); gr.z = __fmaf_rn(s, dz, gr.z);
            float d = __fmul_rn(__fsub_rn(vj.x, vi.x), dx);                  // (v_j - v_i) . (x_i - x_j)
            d = __fmaf_rn(__fsub_rn(vj.y, vi.y), dy, d);
            d = __fmaf_rn(__fsub_rn(vj.z, vi.z), dz, d);
            div = __fmaf_rn(s, d, div);
        }
    }
    // wall ghosts and boundary particles (config), then density, pressure
    // (EOS, or the carried / zeroed PCISPH pressure) and the features
    template <bool BATCH>
    __device__ __forceinline__ void finish(const Params& P, int t, float4 xi, const float4* __restrict__ pos,
                                           const int* __restrict__ list, int cnt, int count, float2* __restrict__ rp,
                                           float* __restrict__ rho_x, int zero_p, float p_scale,
                                           float* __restrict__ feats) {
        if (!REF) {
            ghost_density<BATCH>(P, t, xi, pos, list, cnt, acc);
            if (!BATCH) boundary_density(P, t, xi, acc, P.bnd);
        }
        const float drho = density_deviation(P, acc);
        const float rho = __fadd_rn(P.rho0, drho);
        float p;
        if (P.pci) {
            p = zero_p ? 0.f : rp[t].y;
        } else if (REF) {
            p = P.eos_k * drho;
        } else {
            const float d = drho / P.rho0;
            const float x = 1.f + d;
            const float s = 1.f + x * (1.f + x * (1.f + x * (1.f + x * (1.f + x * (1.f + x)))));
            p = P.eos_k * d * s;
        }
        if (FEAT) {
            div = __fmul_rn(div, -P.k_grad / P.rho0);
            const auto F = faces_of<BATCH>(P, t);
            float dwall = P.hf;
            dwall = fminf(dwall, fminf(xi.x - F.x0(), F.x1() - xi.x));
            dwall = fminf(dwall, fminf(xi.y - F.y0(), F.y1() - xi.y));
            dwall = fminf(dwall, fminf(xi.z - F.z0(), F.z1() - xi.z));
            float4* f = reinterpret_cast<float4*>(feats + (size_t)t * 8);     // two 16-byte stores
            const float adv = __fsub_rn(__fsub_rn(rho, __fmul_rn(__fmul_rn(P.dt, rho), div)), P.rho0);
            const float grad = sqrtf(dist2(gr.x, gr.y, gr.z));
            f[0] = make_float4((float)count * (1.f / 32.f), __fmul_rn(adv / P.rho0, 100.f),
                               __fmul_rn(__fmul_rn(div, P.dt), 100.f),
                               rp[t].y / p_scale);     // the carried pressure, before this pass replaces it
            f[1] = make_float4(__fmul_rn(fmaxf(dwall, 0.f), P.inv_h), __fmul_rn(__fmul_rn(P.k_grad, grad), P.hf) / P.rho0,
                               SMOOTH_P && ws > 0.f ? wp / ws / p_scale : 0.f, 0.f);
        }
        rp[t] = make_float2(rho, p);
        rho_x[t] = rho;
    }
};

template <bool REF, int NF, bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_density_x(Params P, const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, const int* __restrict__ counts,
                                                      const int* __restrict__ list, float2* __restrict__ rp,
                                                      float* __restrict__ rho_x, int zero_p, float p_scale,
                                                      float* __restrict__ feats) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xi = pos[t];
    const int count = counts[t];
    const int cnt = min(count, P.cap);
    DensityX<REF, NF> D;
    D.begin(vel, t);
    for_each_nbr(list, P.n, t, cnt, [&](const int j) { D.pair(P, xi, pos[j], j, vel, rp); });
    D.template finish<BATCH>(P, t, xi, pos, list, cnt, count, rp, rho_x, zero_p, p_scale, feats);
}

// The neighbour build of one scene (config profile) with the density pass
// at x folded in: the 27-cell walk of each particle (walk_neighbours) writes
// its list and, for every neighbour it accepts, adds that pair's density and
// feature terms -- the same terms in the same order as k_density_x over the
// finished list -- so the step saves one sweep over the lists. The ghost
// and boundary terms then walk the list this thread has just written.
template <int NF, int BS>
__global__ void __launch_bounds__(BS) k_build_density(Params P, const float4* __restrict__ pos,
                                                          const float4* __restrict__ vel,
                                                          const uint32_t* __restrict__ keys,
                                                          const uint32_t* __restrict__ cell_start,
                                                          const uint32_t* __restrict__ cell_end,
                                                          int* __restrict__ counts, int* __restrict__ list,
                                                          int* __restrict__ flags, float2* __restrict__ rp,
                                                          float* __restrict__ rho_x, int zero_p, float p_scale,
                                                          float* __restrict__ feats) {
    const int t = blockIdx.x * BS + threadIdx.x;
    const bool valid = t < P.n;     // every lane stays for the warp reductions below
    int cnt = 0;
    if (valid) {
        const float4 pi = pos[t];
        DensityX<false, NF> D;
        D.begin(vel, t);
        int* wq = list + nbr_index(0, P.n, t);
        const size_t qstride = (size_t)4 * (size_t)P.n;
        walk_neighbours<false>(P, t, pi, pos, keys, cell_start, cell_end, [&](uint32_t q, float4 pj) {
            if (cnt < P.cap) {
                wq[cnt & 3] = (int)q;
                D.pair(P, pi, pj, (int)q, vel, rp);
            }
            ++cnt;
            if ((cnt & 3) == 0 && cnt < P.cap) wq += qstride;
        });
        counts[t] = cnt;
        if (cnt > P.cap) atomicOr(&flags[0], 1);
        D.template finish<false>(P, t, pi, pos, list, min(cnt, P.cap), cnt, rp, rho_x, zero_p, p_scale, feats);
    }
    nbr_flags(cnt, flags);
}

// Viscosity (+ reference surface tension) and, when with_pressure, the
// symmetric pressure acceleration, over the list at the start positions.
struct PairSums {
    float3 ap;      // sum (pV_i + pV_j) (1-u)^2 x^_ij   (times k_grad: pressure acceleration)
    float3 fv;      // sum (v_j - v_i) (1-u) / rho_j     (times k_visc: viscosity force density)
    float3 nrm;     // sum x_ij (1-q)^2 / rho_j           (times -k_surf: surface normal)
    float fs;       // sum (1-q)(3-7q) / rho_j           (times -k_surf: surface term)
};

template <bool REF, bool WITH_PRESSURE, bool BATCH = false>
__device__ __forceinline__ PairSums pair_sums(const Params& P, int t, float4 xi, float4 vi, float2 rpi,
                                              const float4* __restrict__ pos, const float4* __restrict__ vel,
                                              const float2* __restrict__ rp, const int* __restrict__ counts,
                                              const int* __restrict__ list) {
    PairSums S;
    S.ap = S.fv = S.nrm = make_float3(0.f, 0.f, 0.f);
    S.fs = 0.f;
    // Config: p/rho0^2 (the PCISPH linearisation; see k_pci_force_predict).
    const float ir0 = 1.f / (P.rho0 * P.rho0);
    const float pVi = WITH_PRESSURE ? (REF ? rpi.y / (rpi.x * rpi.x) : rpi.y * ir0) : 0.f;
    const int cnt = min(counts[t], P.cap);
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        const float4 xj = pos[j];       // the pair's three gathers, ahead of the tests
        const float4 vj = vel[j];
        const float2 rpj = rp[j];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r2 = dist2(dx, dy, dz);
        if (!(r2 > 0.f)) return;
        const float q = r2 * P.inv_h2;
        if (!REF && q >= 1.f) return;
        const float rinv = rsqrtf(r2);
        const float om = 1.f - r2 * rinv * P.inv_h;
        const float inv_rj = 1.f / rpj.x;
        const float sv = om * inv_rj;
        S.fv.x += (vj.x - vi.x) * sv;
        S.fv.y += (vj.y - vi.y) * sv;
        S.fv.z += (vj.z - vi.z) * sv;
        if (WITH_PRESSURE) {
            const float pVj = REF ? rpj.y * inv_rj * inv_rj : rpj.y * ir0;
            const float s = (pVi + pVj) * om * om * rinv;
            S.ap.x += s * dx; S.ap.y += s * dy; S.ap.z += s * dz;
        }
        if (REF) {      // surface tension and normals: reference profile only
            const float t1 = 1.f - q;
            S.fs += t1 * (3.f - 7.f * q) * inv_rj;
            const float sn = t1 * t1 * inv_rj;
            S.nrm.x += dx * sn; S.nrm.y += dy * sn; S.nrm.z += dz * sn;
        }
    });
    if (WITH_PRESSURE && !REF) {
        ghost_pressure<BATCH>(P, t, xi, pVi, pos, (const float*)rp + 1, 2, list, cnt, S.ap);
        if (!BATCH) boundary_pressure(P, t, xi, pVi, S.ap);
    }
    return S;
}

// Non-pressure force density f_v + f_s + rho_i g (the reference's forcesAccum
// is (0, -9.81 rho, 0) in PCISPH, PciSphSystem_Kernel.cu:168, and rho*g from
// ForceExt_Constante in WCSPH, SphSystem.cpp:307-320).
template <bool REF>
__device__ __forceinline__ float3 nonpressure_force(const Params& P, const PairSums& S, float rho) {
    float3 f = make_float3(P.k_visc * S.fv.x, P.k_visc * S.fv.y, P.k_visc * S.fv.z);
    if (REF) {
        const float3 n = make_float3(-P.k_surf * S.nrm.x, -P.k_surf * S.nrm.y, -P.k_surf * S.nrm.z);
        const float ln = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
        if (ln >= P.l) {
            const float c = (-P.k_surf * S.fs) * (-P.sigma) / ln;
            f.x += c * n.x; f.y += c * n.y; f.z += c * n.z;
        }
    }
    f.x += rho * P.gx; f.y += rho * P.gy; f.z += rho * P.gz;
    return f;
}

// WCSPH: forces, leap-frog, walls and velocity interpolation in one sweep.
template <bool REF>
__global__ void __launch_bounds__(kBlock) k_wcsph_force(Params P, const float4* __restrict__ pos,
                                                        const float4* __restrict__ vel, const float4* __restrict__ vap,
                                                        const float2* __restrict__ rp, const int* __restrict__ counts,
                                                        const int* __restrict__ list, float4* __restrict__ pos_out,
                                                        float4* __restrict__ vel_out, float4* __restrict__ vap_out,
                                                        float4* __restrict__ fnp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xi = pos[t], vi = vel[t], vh = vap[t];
    const float2 rpi = rp[t];
    const PairSums S = pair_sums<REF, true>(P, t, xi, vi, rpi, pos, vel, rp, counts, list);
    const float3 f = nonpressure_force<REF>(P, S, rpi.x);
    fnp[t] = make_float4(f.x, f.y, f.z, 0.f);
    const float3 aw = wall_accel<REF>(P, t, xi, vh);
    const float ir = 1.f / rpi.x;
    const float3 a = make_float3(f.x * ir + P.k_grad * S.ap.x + aw.x, f.y * ir + P.k_grad * S.ap.y + aw.y,
                                 f.z * ir + P.k_grad * S.ap.z + aw.z);
    float3 v = make_float3(vh.x + a.x * P.dt, vh.y + a.y * P.dt, vh.z + a.z * P.dt);
    float3 x = make_float3(xi.x + v.x * P.dt, xi.y + v.y * P.dt, xi.z + v.z * P.dt);
    if (REF) box_project(P, t, x, v);   // config WCSPH: penalty walls only
    pos_out[t] = make_float4(x.x, x.y, x.z, 0.f);
    vap_out[t] = make_float4(v.x, v.y, v.z, 0.f);
    vel_out[t] = make_float4((vh.x + v.x) * 0.5f, (vh.y + v.y) * 0.5f, (vh.z + v.z) * 0.5f, 0.f);
}

// PCISPH set-up sweep: non-pressure forces at x (and, for a warm start, the
// pressure acceleration of the carried pressure), then the first prediction.
template <bool REF, bool WARM, bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_pci_init(Params P, const float4* __restrict__ pos,
                                                     const float4* __restrict__ vel, const float4* __restrict__ vap,
                                                     const float2* __restrict__ rp, const int* __restrict__ counts,
                                                     const int* __restrict__ list, float4* __restrict__ fnp,
                                                     float4* __restrict__ xs, float4* __restrict__ vs) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xi = pos[t], vi = vel[t], vh = vap[t];
    const float2 rpi = rp[t];
    const PairSums S = pair_sums<REF, WARM, BATCH>(P, t, xi, vi, rpi, pos, vel, rp, counts, list);
    const float3 f = nonpressure_force<REF>(P, S, rpi.x);
    fnp[t] = make_float4(f.x, f.y, f.z, 0.f);
    const float3 aw = wall_accel<REF, BATCH>(P, t, xi, vh);
    const float ir = 1.f / rpi.x;
    const float ap = WARM ? P.k_grad : 0.f;
    const float3 a = make_float3(f.x * ir + ap * S.ap.x + aw.x, f.y * ir + ap * S.ap.y + aw.y,
                                 f.z * ir + ap * S.ap.z + aw.z);
    const float3 v = make_float3(vh.x + a.x * P.dt, vh.y + a.y * P.dt, vh.z + a.z * P.dt);
    vs[t] = make_float4(v.x, v.y, v.z, 0.f);
    xs[t] = make_float4(xi.x + v.x * P.dt, xi.y + v.y * P.dt, xi.z + v.z * P.dt, 0.f);
}

// PCISPH density pass at x*: rho*, the gradient sums of the pressure
// increment, the candidate pressure and the FP64 max compression error.
// Batch: scenes that have converged are left as they are, and the error is
// the max over each scene (P.err_scene).
// The density pass for sorted particle t (t < P.n, its scene still
// iterating): rho* and the candidate pressure into rpc[t]; returns the
// compression error (rho* - rho0)/rho0 in FP64.
template <bool REF, bool BATCH, class F4, class F2, class F2o>
__device__ __forceinline__ double pci_density_at(const Params& P, int t, F4 xs, F2 rp, const int* __restrict__ counts,
                                                 const int* __restrict__ list, F2o rpc) {
    const float4 xi = xs[t];
    const int cnt = min(counts[t], P.cap);
    Kahan acc;
    float3 T1 = make_float3(0.f, 0.f, 0.f);
    float T2 = 0.f;
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        const float4 xj = xs[j];
        const float dx = __fsub_rn(xi.x, xj.x), dy = __fsub_rn(xi.y, xj.y), dz = __fsub_rn(xi.z, xj.z);
        const float r2 = dist2(dx, dy, dz);
        const float q = __fmul_rn(r2, P.inv_h2);
        if (!REF && q >= 1.f) return;
        add_poly6(acc, q);
        if (REF && r2 > 0.f) {
            const float rinv = rsqrtf(r2);
            const float om = 1.f - r2 * rinv * P.inv_h;
            const float g = om * om;
            const float s = g * rinv;
            T1.x += s * dx; T1.y += s * dy; T1.z += s * dz;
            T2 += g * g;
        }
    });
    if (!REF) {
        ghost_density<BATCH>(P, t, xi, xs, list, cnt, acc);
        if (!BATCH) boundary_density(P, t, xi, acc, P.bnd_pred ? P.bnd_pred : P.bnd);
    }
    const float drho = density_deviation(P, acc);
    const float rho = __fadd_rn(P.rho0, drho);
    float p = rp[t].y;
    if (REF) {              // per-particle factor, compressed particles only
        if (drho > 0.f && T2 > 0.f) p += P.k_press * drho / (T1.x * T1.x + T1.y * T1.y + T1.z * T1.z + T2);
    } else {                // prototype factor, every particle, p >= 0
        p = fmaxf(0.f, __fmaf_rn(P.k_delta, drho, p));
    }
    rpc[t] = make_float2(rho, p);
    return (double)drho / P.rho0_d;
}

// The max of the pass's errors. Batch: per scene (P.err_scene); a warp
// inside one scene reduces first, one straddling two or more reduces per
// lane; sc = the slot's scene, -1 for none. Single scene (the persistent
// corrector, once per block and pass): per block, one ordered-integer atomic
// max into err_slot; every thread of the block calls it.
template <bool BATCH, int BS>
__device__ __forceinline__ void reduce_error(const Params& P, int sc, double err, unsigned long long* err_slot,
                                             double* s_err) {
    if constexpr (BATCH) {
        const int sc0 = __shfl_sync(0xffffffffu, sc, 0);
        if (__all_sync(0xffffffffu, sc == sc0 || sc < 0)) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
            if ((threadIdx.x & 31) == 0 && sc0 >= 0 && err > -1e300) atomicMax(&P.err_scene[sc0], order_double(err));
        } else if (sc >= 0 && err > -1e300) {
            atomicMax(&P.err_scene[sc], order_double(err));
        }
    } else {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if ((threadIdx.x & 31) == 0) s_err[threadIdx.x >> 5] = err;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = s_err[0];
            for (int w = 1; w < BS / 32; ++w) m = fmax(m, s_err[w]);
            if (m > -1e300) atomicMax(err_slot, order_double(m));
        }
        __syncthreads();
    }
}

// PCISPH density pass at x*: rho*, the gradient sums of the pressure
// increment, the candidate pressure and the FP64 max compression error.
// Batch: scenes that have converged are left as they are, and the error is
// the max over each scene (P.err_scene).
// Single scene: the max over each warp, then one ordered-integer atomic max
// per warp (a reduction without return: the warp leaves at once). A block-
// level reduction made the block's early warps wait at its barrier for the
// slowest one, a third of the pass's stall cycles at 1M particles.
template <bool BATCH, int BS>
__device__ __forceinline__ void warp_max_error(const Params& P, int sc, double err, unsigned long long* err_slot) {
    if constexpr (BATCH) {
        reduce_error<true, BS>(P, sc, err, err_slot, nullptr);
    } else {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if ((threadIdx.x & 31) == 0 && err > -1e300) atomicMax(err_slot, order_double(err));
    }
}

template <bool REF, bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_pci_density(Params P, const float4* __restrict__ xs,
                                                        const float2* __restrict__ rp, const int* __restrict__ counts,
                                                        const int* __restrict__ list, float2* __restrict__ rpc,
                                                        unsigned long long* __restrict__ err_slot) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double err = -1e300;
    const int sc = BATCH && t < P.n ? (int)P.slot_scene[t] : -1;
    if (t < P.n && (!BATCH || P.active[sc])) err = pci_density_at<REF, BATCH>(P, t, xs, rp, counts, list, rpc);
    warp_max_error<BATCH, BS>(P, sc, err, err_slot);
}

// PCISPH pressure-force pass fused with the next prediction; commits the
// candidate pressure. Reference profile: at the predicted positions x*, with
// p/rho*^2 (PciSphSystem_Kernel.cu:88-114 runs on the predicted state).
// Config profile: at the step's start positions x, with p/rho0^2. That keeps
// the corrector a linear iteration in p: at x*, x* = x + dt^2 a(x*) is a
// fixed-point iteration in positions whose gain grows with p dt^2/h^2, and
// with rho* in p/rho^2 the force feeds back on the density; under a 0.64 m
// column either one makes the corrector diverge.
// The pressure-force pass for sorted particle t (t < P.n, its scene still
// iterating): the next prediction into xs_next[t] and vs[t], and the
// candidate pressure committed to rp[t].
template <bool REF, bool BATCH, class F4, class F2>
__device__ __forceinline__ void pci_force_at(const Params& P, int t, const float4* __restrict__ pos,
                                             const float4* __restrict__ vap, const float4* __restrict__ fnp, F4 xs,
                                             F2 rpc, const int* __restrict__ counts, const int* __restrict__ list,
                                             float4* xs_next, float4* vs, float2* rp) {
    const float4 xi = REF ? xs[t] : pos[t];
    const float2 ri = rpc[t];
    const float ir0 = 1.f / __fmul_rn(P.rho0, P.rho0);
    const float pVi = REF ? ri.y / __fmul_rn(ri.x, ri.x) : __fmul_rn(ri.y, ir0);
    const int cnt = min(counts[t], P.cap);
    float3 acc = make_float3(0.f, 0.f, 0.f);
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        // both gathers of the pair issue before its distance test, so a pair
        // costs one dependent load after the list, not two
        const float4 xj = REF ? xs[j] : pos[j];
        const float2 rj = rpc[j];
        const float dx = __fsub_rn(xi.x, xj.x), dy = __fsub_rn(xi.y, xj.y), dz = __fsub_rn(xi.z, xj.z);
        const float r2 = dist2(dx, dy, dz);
        if (!(r2 > 0.f)) return;
        if (!REF && __fmul_rn(r2, P.inv_h2) >= 1.f) return;
        const float rinv = rsqrtf(r2);
        const float om = spiky_om(P, r2, rinv);
        // pV_i + pV_j (config: p_j / rho0^2 fused into the sum), then products only
        const float pv = REF ? pVi + rj.y / (rj.x * rj.x) : __fmaf_rn(rj.y, ir0, pVi);
        const float s = pv * om * om * rinv;
        acc.x = __fmaf_rn(s, dx, acc.x); acc.y = __fmaf_rn(s, dy, acc.y); acc.z = __fmaf_rn(s, dz, acc.z);
    });
    if (!REF) {
        ghost_pressure<BATCH>(P, t, xi, pVi, pos, (const float*)&rpc[0] + 1, 2, list, cnt, acc);
        if (!BATCH) boundary_pressure(P, t, xi, pVi, acc);
    }
    const float4 x0 = pos[t], vh = vap[t], f = fnp[t];
    const float3 aw = wall_accel<REF, BATCH>(P, t, x0, vh);
    const float ir = 1.f / ri.x;
    auto accel = [&](float fc, float ac, float wc) {     // f/rho + k_grad sum + wall
        return __fadd_rn(__fmaf_rn(P.k_grad, ac, __fmul_rn(fc, ir)), wc);
    };
    const float3 a = make_float3(accel(f.x, acc.x, aw.x), accel(f.y, acc.y, aw.y), accel(f.z, acc.z, aw.z));
    const float3 v = make_float3(__fmaf_rn(a.x, P.dt, vh.x), __fmaf_rn(a.y, P.dt, vh.y), __fmaf_rn(a.z, P.dt, vh.z));
    vs[t] = make_float4(v.x, v.y, v.z, 0.f);
    xs_next[t] = make_float4(__fmaf_rn(v.x, P.dt, x0.x), __fmaf_rn(v.y, P.dt, x0.y), __fmaf_rn(v.z, P.dt, x0.z), 0.f);
    rp[t] = ri;
}

// PCISPH pressure-force pass fused with the next prediction; commits the
// candidate pressure. Reference profile: at the predicted positions x*, with
// p/rho*^2 (PciSphSystem_Kernel.cu:88-114 runs on the predicted state).
// Config profile: at the step's start positions x, with p/rho0^2. That keeps
// the corrector a linear iteration in p: at x*, x* = x + dt^2 a(x*) is a
// fixed-point iteration in positions whose gain grows with p dt^2/h^2, and
// with rho* in p/rho^2 the force feeds back on the density; under a 0.64 m
// column either one makes the corrector diverge.
template <bool REF, bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_pci_force_predict(Params P, const float4* __restrict__ pos,
                                                              const float4* __restrict__ vap,
                                                              const float4* __restrict__ fnp,
                                                              const float4* __restrict__ xs,
                                                              const float2* __restrict__ rpc,
                                                              const int* __restrict__ counts,
                                                              const int* __restrict__ list, float4* __restrict__ xs_next,
                                                              float4* __restrict__ vs, float2* __restrict__ rp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    if (BATCH && !P.active[P.slot_scene[t]]) return;     // its scene has converged
    if (!BATCH && P.active && !P.active[0]) return;      // single scene, corrector decided on the device: converged
    pci_force_at<REF, BATCH>(P, t, pos, vap, fnp, xs, rpc, counts, list, xs_next, vs, rp);
}

// The whole corrector loop of a config-profile scene or batch in one
// cooperative launch: every block strides over the particles, and grid-wide
// barriers separate {density pass, decision, pressure-force pass} as kernel
// boundaries do in the graph. Block 0 takes the decision (the batch's rule,
// corrector_decide). The arrays that the passes write and the next pass
// reads (x*, the pressures, the decision's words) are read through plain
// pointers here, not the read-only path: the barrier's acquire makes other
// blocks' writes visible to ordinary loads. Same passes, same order, same
// arithmetic as the graph's loop: the results are bit-identical.
// Five resident blocks of 256 per SM (at most 48 registers, no spills),
// the occupancy of the separate pressure-force pass.
template <bool BATCH, int BS>
__global__ void __launch_bounds__(BS, 5) k_corrector_persistent(Params P, const float4* __restrict__ pos,
                                                                 const float4* __restrict__ vap,
                                                                 const float4* __restrict__ fnp, float4* xs, float2* rp,
                                                                 float2* rpc, const int* __restrict__ counts,
                                                                 const int* __restrict__ list, float4* vs,
                                                                 unsigned long long* err_slot, int S, int min_it,
                                                                 int max_it, double eta, uint8_t* active,
                                                                 unsigned long long* err_scene,
                                                                 unsigned long long* err_hist, int* loop) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double s_err[BS / 32];
    __shared__ int s_any;
    const long long stride = (long long)gridDim.x * BS;
    if (blockIdx.x == 0) corrector_begin(S, max_it, active, err_scene, err_hist, (PSB_MAX_ITERS + 1) * S, loop);
    grid.sync();
    for (int pass = 0; pass < max_it; ++pass) {
        // density pass (warp-uniform bounds: the reduction is warp-synchronous)
        double emax = -1e300;
        for (long long base = (long long)blockIdx.x * BS; base < P.n; base += stride) {
            const int t = (int)(base + threadIdx.x);
            double err = -1e300;
            const int sc = BATCH && t < P.n ? (int)P.slot_scene[t] : -1;
            const volatile uint8_t* act = active;
            if (t < P.n && (!BATCH || act[sc])) err = pci_density_at<false, BATCH>(P, t, (const float4*)xs, (const float2*)rp, counts, list, rpc);
            if (BATCH) reduce_error<true, BS>(P, sc, err, err_slot, s_err);
            else emax = fmax(emax, err);
        }
        if (!BATCH) reduce_error<false, BS>(P, -1, emax, err_slot, s_err);
        grid.sync();
        if (blockIdx.x == 0) corrector_decide(S, min_it, max_it, eta, active, err_scene, err_hist, loop, &s_any);
        grid.sync();
        const int cont = *(volatile int*)&loop[1];
        // pressure-force pass and the next prediction, x* in place
        for (long long base = (long long)blockIdx.x * BS; base < P.n; base += stride) {
            const int t = (int)(base + threadIdx.x);
            if (t >= P.n) continue;
            const volatile uint8_t* act = active;
            if (!act[BATCH ? (int)P.slot_scene[t] : 0]) continue;
            pci_force_at<false, BATCH>(P, t, pos, vap, fnp, (const float4*)xs, (const float2*)rpc, counts, list, xs,
                                       vs, rp);
        }
        if (!cont) break;
        grid.sync();
    }
}

// Commit of the last prediction, walls, collision objects (COLL: the start
// position pos[t] is read before it is overwritten), velocity interpolation.
template <bool BATCH, bool COLL>
__global__ void __launch_bounds__(kBlock) k_pci_commit(Params P, const float4* __restrict__ xs,
                                                       const float4* __restrict__ vs, const float2* __restrict__ rpc,
                                                       int have_density_pass, float4* __restrict__ pos,
                                                       float4* __restrict__ vel, float4* __restrict__ vap,
                                                       float2* __restrict__ rp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    float3 x = f3(xs[t]), v = f3(vs[t]);
    const float4 vh = vap[t];
    box_project<BATCH>(P, t, x, v);
    if constexpr (COLL) {
        const float4 x0 = pos[t];
        coll::V3<float> cx{x.x, x.y, x.z}, cv{v.x, v.y, v.z};
        coll::apply_colliders(P.coll, P.n_coll, P.dt, coll::V3<float>{x0.x, x0.y, x0.z}, cx, cv);
        x = make_float3(cx.x, cx.y, cx.z);
        v = make_float3(cv.x, cv.y, cv.z);
    }
    pos[t] = make_float4(x.x, x.y, x.z, 0.f);
    vap[t] = make_float4(v.x, v.y, v.z, 0.f);
    vel[t] = make_float4((vh.x + v.x) * 0.5f, (vh.y + v.y) * 0.5f, (vh.z + v.z) * 0.5f, 0.f);
    if (have_density_pass) rp[t].x = rpc[t].x;
}

// XSPH velocity smoothing (Monaghan 1989) of the committed prediction,
// config PCISPH: v_i + xsph sum_j (m/rho0) W_ij (v_j - v_i) over the list at
// x*, W the poly6 kernel (m W = k_rho (1-q)^3). Positions are not moved.
template <int BS>
__global__ void __launch_bounds__(BS) k_xsph(Params P, const float4* __restrict__ xs,
                                                 const float4* __restrict__ vs, const int* __restrict__ counts,
                                                 const int* __restrict__ list, float4* __restrict__ vs_out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const float4 xi = xs[t], vi = vs[t];
    const int cnt = min(counts[t], P.cap);
    float3 dv = make_float3(0.f, 0.f, 0.f);
    for_each_nbr(list, P.n, t, cnt, [&](const int j) {
        const float4 xj = xs[j];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float q = dist2(dx, dy, dz) * P.inv_h2;
        if (q >= 1.f) return;
        const float4 vj = vs[j];
        const float w = (1.f - q) * (1.f - q) * (1.f - q);
        dv.x += w * (vj.x - vi.x); dv.y += w * (vj.y - vi.y); dv.z += w * (vj.z - vi.z);
    });
    vs_out[t] = make_float4(vi.x + P.xsph_k * dv.x, vi.y + P.xsph_k * dv.y, vi.z + P.xsph_k * dv.z, 0.f);
}

inline int grid_of(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

// Kernels are specialised on the physics profile (REF), on batching
// (P.scenes set: per-scene boxes and convergence; config profile only) and
// on the tuned block size.
template <int BS>
inline unsigned blocks_of(int n) { return (unsigned)((n + BS - 1) / BS); }


void launch_density_x(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                      const int* list, float2* rp, float* rho_x, int zero_p, float p_scale, float* feats, int nfeat) {
    if (P.n <= 0) return;
    with_block(P.tune.density_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        auto go = [&](auto kernel) {
            kernel<<<blocks_of<BS>(P.n), BS, 0, st>>>(P, pos, vel, counts, list, rp, rho_x, zero_p, p_scale, feats);
        };
        const int nf = feats ? (nfeat > 6 ? 7 : 6) : 0;
        if (P.ref) go(k_density_x<true, 0, false, BS>);
        else if (P.scenes) {
            if (nf == 7) go(k_density_x<false, 7, true, BS>);
            else if (nf == 6) go(k_density_x<false, 6, true, BS>);
            else go(k_density_x<false, 0, true, BS>);
        } else if (nf == 7) go(k_density_x<false, 7, false, BS>);
        else if (nf == 6) go(k_density_x<false, 6, false, BS>);
        else go(k_density_x<false, 0, false, BS>);
    });
}

void launch_build_density(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const uint32_t* keys,
                          const uint32_t* cell_start, const uint32_t* cell_end, int* counts, int* list, int* flags,
                          float2* rp, float* rho_x, int zero_p, float p_scale, float* feats, int nfeat) {
    if (P.n <= 0) return;
    with_block(P.tune.nbr_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        auto go = [&](auto kernel) {
            kernel<<<blocks_of<BS>(P.n), BS, 0, st>>>(P, pos, vel, keys, cell_start, cell_end, counts, list, flags, rp,
                                                      rho_x, zero_p, p_scale, feats);
        };
        const int nf = feats ? (nfeat > 6 ? 7 : 6) : 0;
        if (nf == 7) go(k_build_density<7, BS>);
        else if (nf == 6) go(k_build_density<6, BS>);
        else go(k_build_density<0, BS>);
    });
}

void launch_wcsph_force(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const float4* vap,
                        const float2* rp, const int* counts, const int* list, float4* pos_out, float4* vel_out,
                        float4* vap_out, float4* fnp) {
    if (P.n <= 0) return;
    if (P.ref)
        k_wcsph_force<true><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, vap, rp, counts, list, pos_out, vel_out,
                                                             vap_out, fnp);
    else
        k_wcsph_force<false><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, vel, vap, rp, counts, list, pos_out, vel_out,
                                                              vap_out, fnp);
}

void launch_pci_init(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const float4* vap,
                     const float2* rp, const int* counts, const int* list, int warm, float4* fnp, float4* xs,
                     float4* vs) {
    if (P.n <= 0) return;
    with_block(P.tune.init_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        auto go = [&](auto kernel) {
            kernel<<<blocks_of<BS>(P.n), BS, 0, st>>>(P, pos, vel, vap, rp, counts, list, fnp, xs, vs);
        };
        if (P.ref) { if (warm) go(k_pci_init<true, true, false, BS>); else go(k_pci_init<true, false, false, BS>); }
        else if (P.scenes) { if (warm) go(k_pci_init<false, true, true, BS>); else go(k_pci_init<false, false, true, BS>); }
        else if (warm) go(k_pci_init<false, true, false, BS>);
        else go(k_pci_init<false, false, false, BS>);
    });
}

void launch_pci_density(cudaStream_t st, const Params& P, const float4* xs, const float2* rp, const int* counts,
                        const int* list, float2* rpc, unsigned long long* err_slot) {
    if (P.n <= 0) return;
    with_block(P.tune.pci_density_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        auto go = [&](auto kernel) {
            kernel<<<blocks_of<BS>(P.n), BS, 0, st>>>(P, xs, rp, counts, list, rpc, err_slot);
        };
        if (P.ref) go(k_pci_density<true, false, BS>);
        else if (P.scenes) go(k_pci_density<false, true, BS>);
        else go(k_pci_density<false, false, BS>);
    });
}

cudaError_t launch_corrector_persistent(cudaStream_t st, const Params& P, const float4* pos, const float4* vap,
                                        const float4* fnp, float4* xs, float2* rp, float2* rpc, const int* counts,
                                        const int* list, float4* vs, int S, int min_it, int max_it, double eta,
                                        uint8_t* active, unsigned long long* err_scene, unsigned long long* err_hist,
                                        int* loop) {
    constexpr int BS = 256;
    auto go = [&](auto kernel) -> cudaError_t {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, BS, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
        // every block resident at once (the grid barrier needs it), no more
        // blocks than the particles fill
        const long long need = ((long long)P.n + BS - 1) / BS;
        const int grid = (int)std::max(1LL, std::min<long long>((long long)per_sm * sms, need));
        unsigned long long* err_slot = err_scene;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(BS);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kernel, P, pos, vap, fnp, xs, rp, rpc, counts, list, vs, err_slot, S, min_it,
                                  max_it, eta, active, err_scene, err_hist, loop);
    };
    if (P.ref) return cudaErrorInvalidValue;
    return P.scenes ? go(k_corrector_persistent<true, BS>) : go(k_corrector_persistent<false, BS>);
}
void launch_pci_force_predict(cudaStream_t st, const Params& P, const float4* pos, const float4* vap,
                              const float4* fnp, const float4* xs, const float2* rpc, const int* counts,
                              const int* list, float4* xs_next, float4* vs, float2* rp) {
    if (P.n <= 0) return;
    with_block(P.tune.force_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        auto go = [&](auto kernel) {
            kernel<<<blocks_of<BS>(P.n), BS, 0, st>>>(P, pos, vap, fnp, xs, rpc, counts, list, xs_next, vs, rp);
        };
        if (P.ref) go(k_pci_force_predict<true, false, BS>);
        else if (P.scenes) go(k_pci_force_predict<false, true, BS>);
        else go(k_pci_force_predict<false, false, BS>);
    });
}

void launch_xsph(cudaStream_t st, const Params& P, const float4* xs, const float4* vs, const int* counts,
                 const int* list, float4* vs_out) {
    if (P.n <= 0) return;
    with_block(P.tune.xsph_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        k_xsph<BS><<<blocks_of<BS>(P.n), BS, 0, st>>>(P, xs, vs, counts, list, vs_out);
    });
}

void launch_pci_commit(cudaStream_t st, const Params& P, const float4* xs, const float4* vs, const float2* rpc,
                       int have_density_pass, float4* pos, float4* vel, float4* vap, float2* rp) {
    if (P.n <= 0) return;
    if (P.scenes)
        k_pci_commit<true, false><<<grid_of(P.n), kBlock, 0, st>>>(P, xs, vs, rpc, have_density_pass, pos, vel, vap, rp);
    else if (P.n_coll > 0)
        k_pci_commit<false, true><<<grid_of(P.n), kBlock, 0, st>>>(P, xs, vs, rpc, have_density_pass, pos, vel, vap, rp);
    else k_pci_commit<false, false><<<grid_of(P.n), kBlock, 0, st>>>(P, xs, vs, rpc, have_density_pass, pos, vel, vap, rp);
}

}  // namespace psb
