/*
 * psb_oracle.c -- FP64 CPU restatement of the PSB particle-simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU path and the "port" CPU
 * baseline. Only tests/, the smoke check and bench.py's CPU-baseline leg use
 * it; the product never links it.
 *
 * Reference-compatible profile (ORC_PROFILE_REF): each formula below is the
 * reference's, restated term by term with the same association order so the
 * results agree with the reference kernels run on the CPU (oracle/_ref) to
 * ~1e-12 relative. Sources (paths inside the reference project):
 *   cell index ............ src/Utils/Neighborhood/UniformGrid/UniformGridKernel.cu:43-55
 *   neighbour test ........ UniformGridKernel.cu:58-95 (sqrt(d.d) <= h_i, self included)
 *   WCSPH density/EOS ..... src/Kernel/System/Fluid_System/SPHSystem/SPH/SphKernel.cu:9-27
 *   WCSPH forces .......... SphKernel.cu:32-91
 *   gravity (force dens.) . src/Kernel/ForcesExt/Constante/ForceExt_Constante.cu:15-23
 *   leap-frog ............. SphKernel.cu:95-124, interpolation SphKernel.cu:128-135
 *   PCISPH density ........ .../PCISPH/PciSphSystem_Kernel.cu:70-85
 *   PCISPH non-pressure ... PciSphSystem_Kernel.cu:117-170 (p <- 0, sigma <- 0.0728, g = -9.81 y)
 *   PCISPH pressure update  PciSphSystem_Kernel.cu:36-67
 *   PCISPH pressure force . PciSphSystem_Kernel.cu:88-114
 *   PCISPH sequence ....... .../PCISPH/PciSphSystem.cu:8-68, PciSphSystem.cpp:163-204
 *   box walls ............. src/Kernel/Collision/BoxCollision/BoxCollision_Kernel.cu:7-34
 *   collision objects ..... src/Kernel/Collision/* (see orc_collide), after the box,
 *                           Collision.cpp:44-49
 *   DEM contacts .......... src/Kernel/System/SimpleSystem/CudaParticle_Kernel.cu:10-55 (as executed,
 *                           see dem_pair_ref), integrateEuler ParticleKernel.cu:12-20,
 *                           sequence CudaSystem.cpp:207-224
 * The reference's predict-then-restore passes are restated as a predict that
 * leaves the saved state untouched; the values are the same.
 *
 * Config profile (ORC_PROFILE_CONFIG): the scene text's method -- Tait EOS,
 * penalty walls, eta-controlled corrector loop with min/max iterations, no
 * surface tension, kernels cut off at r >= h. No reference counterpart.
 */
#include "psb_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846

/* Storage rounding: with float_state the oracle keeps every stored array in
 * float, at the same points the GPU path stores FP32. */
#define RND(P, x) ((P)->float_state ? (double)(float)(x) : (x))

uint64_t orc_splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void orc_lattice(const int32_t nxyz[3], double spacing, const double origin[3], double jitter,
                 uint64_t seed, int32_t id0, float* pos3) {
    const int64_t n = (int64_t)nxyz[0] * nxyz[1] * nxyz[2];
    for (int64_t id = 0; id < n; ++id) {
        const int64_t ijk[3] = {id % nxyz[0], (id / nxyz[0]) % nxyz[1], id / ((int64_t)nxyz[0] * nxyz[1])};
        for (int a = 0; a < 3; ++a) {
            const uint64_t z = orc_splitmix64(seed ^ ((uint64_t)(id + id0) * 3u + (uint64_t)a));
            const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);   /* [0,1) */
            const double j = jitter * (2.0 * u - 1.0);
            const double x = origin[a] + ((double)ijk[a] + 0.5) * spacing + j;
            pos3[3 * id + a] = (float)x;
        }
    }
}

/* Clamped into [0, dim-1] in double before the conversion to int, so that
 * infinities, NaN and huge coordinates land in the border cells. */
static inline int cell_coord(double x, float mn, float cell, int dim, int* clamped) {
    const double t = floor((x - (double)mn) / (double)cell);
    if (!(t >= 0.0)) { *clamped = 1; return 0; }
    if (t >= (double)dim) { *clamped = 1; return dim - 1; }
    return (int)t;
}

void orc_cell_keys(int32_t n, const double* pos, const float grid_min[3], float cell, const int32_t dims[3],
                   uint32_t* keys, int32_t* nclamped) {
    int32_t cl = 0;
#pragma omp parallel for reduction(+ : cl) schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        int c = 0;
        const int a = cell_coord(pos[3 * i + 0], grid_min[0], cell, dims[0], &c);
        const int b = cell_coord(pos[3 * i + 1], grid_min[1], cell, dims[1], &c);
        const int d = cell_coord(pos[3 * i + 2], grid_min[2], cell, dims[2], &c);
        keys[i] = (uint32_t)a + (uint32_t)b * (uint32_t)dims[0] + (uint32_t)d * (uint32_t)dims[0] * (uint32_t)dims[1];
        cl += c;
    }
    if (nclamped) *nclamped = cl;
}

/* Counting sort over the cell range: stable, so ties keep increasing id. */
static void sort_by_key(int32_t n, const uint32_t* keys, uint32_t ncells, int32_t* perm, int32_t* start /* ncells+1 */) {
    memset(start, 0, sizeof(int32_t) * ((size_t)ncells + 1));
    for (int32_t i = 0; i < n; ++i) start[keys[i] + 1]++;
    for (uint32_t c = 0; c < ncells; ++c) start[c + 1] += start[c];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * ((size_t)ncells + 1));
    memcpy(fill, start, sizeof(int32_t) * ((size_t)ncells + 1));
    for (int32_t i = 0; i < n; ++i) perm[fill[keys[i]]++] = i;
    free(fill);
}

void orc_sort_perm(int32_t n, const uint32_t* keys, int32_t* perm) {
    uint32_t mx = 0;
    for (int32_t i = 0; i < n; ++i) mx = keys[i] > mx ? keys[i] : mx;
    int32_t* start = (int32_t*)malloc(sizeof(int32_t) * ((size_t)mx + 2));
    sort_by_key(n, keys, mx + 1, perm, start);
    free(start);
}

/* Reference neighbour test: length(x_i - x_j) <= radius_i, evaluated as
 * sqrt((dx*dx + dy*dy) + dz*dz) in double (double3.h:15-47). */
static inline int is_neighbor(const double* xi, const double* xj, double h) {
    const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    return sqrt(dx * dx + dy * dy + dz * dz) <= h;
}

int64_t orc_neighbors(const orc_params* P, const double* pos, int32_t cap, int32_t* counts, int32_t* list) {
    const int32_t n = P->n;
    const uint32_t ncells = (uint32_t)P->dims[0] * (uint32_t)P->dims[1] * (uint32_t)P->dims[2];
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* start = (int32_t*)malloc(sizeof(int32_t) * ((size_t)ncells + 1));
    orc_cell_keys(n, pos, P->grid_min, P->cell, P->dims, keys, NULL);
    sort_by_key(n, keys, ncells, perm, start);
    const int nx = P->dims[0], ny = P->dims[1], nz = P->dims[2];
    /* list cut-off: h, or (1 + skin) h in the config profile */
    const double hl = P->profile == ORC_PROFILE_CONFIG ? P->h * (1.0 + P->skin) : P->h;
    int64_t total = 0;
    int overflow = 0;
#pragma omp parallel for reduction(+ : total) reduction(| : overflow) schedule(dynamic, 256)
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t key = keys[i];
        const int ci = (int)(key % (uint32_t)nx), cj = (int)((key / (uint32_t)nx) % (uint32_t)ny),
                  ck = (int)(key / ((uint32_t)nx * (uint32_t)ny));
        int32_t cnt = 0;
        /* z outer, x inner: cells, and so candidates, come in increasing (key, id). */
        for (int k = ck - 1; k <= ck + 1; ++k) {
            if (k < 0 || k >= nz) continue;
            for (int j = cj - 1; j <= cj + 1; ++j) {
                if (j < 0 || j >= ny) continue;
                for (int a = ci - 1; a <= ci + 1; ++a) {
                    if (a < 0 || a >= nx) continue;
                    const uint32_t c = (uint32_t)a + (uint32_t)j * nx + (uint32_t)k * nx * ny;
                    for (int32_t t = start[c]; t < start[c + 1]; ++t) {
                        const int32_t jd = perm[t];
                        if (is_neighbor(&pos[3 * (size_t)i], &pos[3 * (size_t)jd], hl)) {
                            if (list) {
                                if (cnt < cap) list[(size_t)i * cap + cnt] = jd;
                                else overflow = 1;
                            }
                            cnt++;
                        }
                    }
                }
            }
        }
        counts[i] = cnt;
        total += cnt;
    }
    free(keys);
    free(perm);
    free(start);
    return overflow ? -1 : total;
}

static inline double len3(const double* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static inline double dmax(double a, double b) { return a > b ? a : b; }

/* ---- config-profile wall boundary: mirror ghost particles ---------------
 * Every box face within h of a particle reflects the particle's neighbours:
 * for each neighbour j and each non-empty set S of faces that both i and j
 * lie within h of, the ghost x_j^S is x_j reflected across every face in S,
 * with j's pressure and density (Libersky et al. 1993; Colagrossi &
 * Landrini 2003). A ghost can only lie within h of i if j does (reflection
 * moves a point away from the particles on the wall's own side), so i's
 * neighbour list -- self included -- yields every ghost. At a flat wall the
 * ghosts continue the fluid exactly: a uniform pressure exerts no net force
 * and the rest lattice keeps its rest density up to the wall. */
typedef struct { int n; int axis[3]; double plane[3]; double nrm[3]; } walls_t;

static void near_walls(const orc_params* P, const double* x, walls_t* w) {
    const double h = P->h;
    w->n = 0;
    for (int e = 0; e < 3; ++e) {
        const double lo = (double)P->box_min[e], hi = (double)P->box_max[e];
        if (x[e] - lo < h) { w->axis[w->n] = e; w->plane[w->n] = lo; w->nrm[w->n] = 1.0; w->n++; }
        else if (hi - x[e] < h) { w->axis[w->n] = e; w->plane[w->n] = hi; w->nrm[w->n] = -1.0; w->n++; }
    }
}

/* x_i minus the ghost of x_j across the faces of subset `mask` (bit k = face
 * k of w), written to dv. With d = n.(x - plane) the distances on the box
 * side (n the inward normal), the reflected component is n (d_i + d_j), both
 * clamped at 0: a particle pushed through a face still sees its ghosts on
 * the wall side. dpg gets the ghost's hydrostatic pressure offset
 * rho0 (-g.n) 2 d_j per face. Returns 0 when x_j is h or more inside. */
static int ghost(const orc_params* P, const walls_t* w, int mask, const double* xi, const double* xj, double h,
                 double* dv, double* dpg) {
    dv[0] = xi[0] - xj[0]; dv[1] = xi[1] - xj[1]; dv[2] = xi[2] - xj[2];
    *dpg = 0.0;
    for (int k = 0; k < w->n; ++k) {
        if (!(mask >> k & 1)) continue;
        const int e = w->axis[k];
        const double nrm = w->nrm[k];
        double dj = nrm * (xj[e] - w->plane[k]);
        if (dj < 0) dj = 0;
        if (dj >= h) return 0;
        double di = nrm * (xi[e] - w->plane[k]);
        if (di < 0) di = 0;
        dv[e] = nrm * (di + dj);
        *dpg += P->rho0 * (-(double)P->gravity[e] * nrm) * 2.0 * dj;
    }
    return 1;
}

/* ---- config-profile boundary particles (Akinci et al. 2012) ----------------
 * A solid is sampled by particles b of volume psi_b / rho0, with psi_b =
 * rho0 / sum_k W_bk over the boundary particles (eq. 5), so that a sparse or
 * thin sampling still contributes a full kernel's worth of density. A fluid
 * particle i gains sum_b psi_b W_ib in density (eq. 6) and the pressure force
 * -m_i sum_b psi_b (p_i/rho0^2) gradW_ib (eq. 10 with the config profile's
 * rho0 in place of rho_i): the fluid's own pressure mirrored onto the solid.
 * Free slip: no viscous term. Brute force over all b: test sizes only. */
static inline double poly6(double h, double d) { return (315 / (64 * PI_D * pow(h, 9))) * pow((h * h) - (d * d), 3); }

void orc_boundary_psi(const orc_params* P, int32_t nb, const double* bpos, double* psi) {
    const double h = P->h;
#pragma omp parallel for schedule(static)
    for (int32_t b = 0; b < nb; ++b) {
        double s = 0.0;
        for (int32_t k = 0; k < nb; ++k) {
            const double dv[3] = {bpos[3 * b] - bpos[3 * k], bpos[3 * b + 1] - bpos[3 * k + 1],
                                  bpos[3 * b + 2] - bpos[3 * k + 2]};
            const double d = len3(dv);
            if (d < h) s += poly6(h, d);
        }
        psi[b] = P->rho0 / s;
    }
}

/* The boundary particles particle i interacts with: its list, built at the
 * step's start positions within the list cut-off (as the fluid lists are),
 * or all of them when no lists are set. */
static inline int32_t bnd_count(const orc_params* P, int32_t i) {
    return P->bnd_counts ? P->bnd_counts[i] : P->n_bnd;
}
static inline int32_t bnd_at(const orc_params* P, int32_t i, int32_t t) {
    return P->bnd_counts ? P->bnd_lists[(size_t)i * P->bnd_cap + t] : t;
}

static double boundary_density(const orc_params* P, int32_t i, const double* x) {
    double s = 0.0;
    for (int32_t t = 0; t < bnd_count(P, i); ++t) {
        const int32_t b = bnd_at(P, i, t);
        const double dv[3] = {x[0] - P->bnd_pos[3 * b], x[1] - P->bnd_pos[3 * b + 1], x[2] - P->bnd_pos[3 * b + 2]};
        const double d = len3(dv);
        if (d < P->h) s += poly6(P->h, d) * P->bnd_psi[b];
    }
    return s;
}

/* Boundary lists at pos: every boundary particle within the list cut-off
 * (1 + skin) h, inclusive, in index order. */
static void build_bnd_lists(const orc_params* P, const double* pos, int32_t** counts_out, int32_t** lists_out,
                            int32_t* cap_out) {
    const int32_t n = P->n;
    const double hl = P->profile == ORC_PROFILE_CONFIG ? P->h * (1.0 + P->skin) : P->h;
    int32_t* counts = (int32_t*)calloc((size_t)n, sizeof(int32_t));
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        int32_t c = 0;
        for (int32_t b = 0; b < P->n_bnd; ++b) {
            const double dv[3] = {pos[3 * i] - P->bnd_pos[3 * b], pos[3 * i + 1] - P->bnd_pos[3 * b + 1],
                                  pos[3 * i + 2] - P->bnd_pos[3 * b + 2]};
            if (len3(dv) <= hl) ++c;
        }
        counts[i] = c;
    }
    int32_t cap = 1;
    for (int32_t i = 0; i < n; ++i) cap = counts[i] > cap ? counts[i] : cap;
    int32_t* lists = (int32_t*)malloc(sizeof(int32_t) * (size_t)n * (size_t)cap);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        int32_t c = 0;
        for (int32_t b = 0; b < P->n_bnd; ++b) {
            const double dv[3] = {pos[3 * i] - P->bnd_pos[3 * b], pos[3 * i + 1] - P->bnd_pos[3 * b + 1],
                                  pos[3 * i + 2] - P->bnd_pos[3 * b + 2]};
            if (len3(dv) <= hl) lists[(size_t)i * cap + c++] = b;
        }
    }
    *counts_out = counts;
    *lists_out = lists;
    *cap_out = cap;
}

/* Poly6 density term; reference form of compute_Density_PCI (PciSphSystem_Kernel.cu:79-81). */
void orc_density(const orc_params* P, const double* pos, const int32_t* counts, const int32_t* list, int32_t cap,
                 int clamp, double* rho) {
    const double h = P->h, m = P->mass;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < P->n; ++i) {
        double s = 0.0;
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            double dv[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            const double d = len3(dv);
            if (clamp && d >= h) continue;
            s += (315 / (64 * PI_D * pow(h, 9))) * pow((h * h) - (d * d), 3) * m;
        }
        if (clamp) {
            walls_t w;
            near_walls(P, &pos[3 * i], &w);
            for (int mask = 1; mask < (1 << w.n); ++mask)
                for (int32_t t = 0; t < counts[i]; ++t) {
                    const int32_t j = list[(size_t)i * cap + t];
                    double dv[3], dpg;
                    if (!ghost(P, &w, mask, &pos[3 * i], &pos[3 * j], h, dv, &dpg)) continue;
                    const double d = len3(dv);
                    if (d >= h) continue;
                    s += (315 / (64 * PI_D * pow(h, 9))) * pow((h * h) - (d * d), 3) * m;
                }
            if (P->n_bnd > 0) s += boundary_density(P, i, &pos[3 * i]);
        }
        rho[i] = RND(P, s);
    }
}

/* ---- per-pair sweeps ------------------------------------------------------ */

/* Non-pressure force density at (pos, vel, rho). Reference profile, PCISPH:
 * compute_Viscosity_SurfaceTension_Force_PCI (PciSphSystem_Kernel.cu:117-170).
 * Reference profile, WCSPH: the viscosity and surface terms of internalForces
 * (SphKernel.cu:32-91) plus the constant force with rho as mass
 * (ForceExt_Constante.cu:15-23). Config: viscosity + rho*g. */
static void nonpressure_forces(const orc_params* P, const double* pos, const double* vel, const double* rho,
                               const int32_t* counts, const int32_t* list, int32_t cap, double* f) {
    const double h = P->h, m = P->mass, mu = P->mu;
    const int ref = P->profile == ORC_PROFILE_REF, pci = P->method == ORC_PCISPH;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < P->n; ++i) {
        double fv[3] = {0, 0, 0}, nrm[3] = {0, 0, 0}, fsurf = 0.0;
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            const double dv[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            const double d = len3(dv);
            if (!(d > 0)) continue;
            if (!ref && d >= h) continue;
            const double a = PI_D * pow(h, 6);
            const double m_m = 45 * (h - d) / a;
            const double c = (mu + mu) / 2;
            const double inv_rho = 1.0 / rho[j];
            for (int e = 0; e < 3; ++e) fv[e] = fv[e] + c * (vel[3 * j + e] - vel[3 * i + e]) * m * m_m * inv_rho;
            if (ref) {
                const double b = 32 * PI_D * (double)powf((float)h, 9.0f);
                const double m_d = -(945 / b) * ((h * h) - (d * d)) * ((3 * h * h) - (7 * d * d));
                fsurf += m_d * (m / rho[j]);
                const double aN = pci ? 32 * PI_D * pow(h, 9) : b;
                const double mk = -945 / aN;
                const double w2 = pow((h * h) - (d * d), 2);
                for (int e = 0; e < 3; ++e) nrm[e] = nrm[e] + dv[e] * (m / rho[j]) * w2 * mk;
            }
        }
        double fs[3] = {0, 0, 0};
        if (ref) {
            const double lN = len3(nrm);
            if (lN >= P->l) {
                const double sigma = pci ? 0.0728 : P->sigma;
                const double inv = 1.0 / lN;
                for (int e = 0; e < 3; ++e) fs[e] = fsurf * (-sigma) * nrm[e] * inv;
            }
        }
        double g[3];
        if (ref && pci) {
            g[0] = 0.0; g[1] = -9.81 * rho[i]; g[2] = 0.0;     /* forcesAccum, PciSphSystem_Kernel.cu:168 */
        } else {
            for (int e = 0; e < 3; ++e) g[e] = (double)P->gravity[e] * rho[i];
        }
        for (int e = 0; e < 3; ++e) f[3 * i + e] = RND(P, (g[e] + fv[e]) + fs[e]);
    }
}

/* Symmetric spiky pressure force density -rho_i sum m (p_i/rho_i^2 + p_j/rho_j^2) gradW
 * (SphKernel.cu:53-61,79; PciSphSystem_Kernel.cu:96-112). */
static void pressure_forces(const orc_params* P, const double* pos, const double* rho, const double* p,
                            const int32_t* counts, const int32_t* list, int32_t cap, double* fp) {
    const double h = P->h, m = P->mass;
    const int clamp = P->profile == ORC_PROFILE_CONFIG;
    /* Config: p/rho0^2 (Solenthaler & Pajarola 2009 approximate rho by rho0
     * in the pressure force, which keeps the corrector linear in p; with the
     * predicted density there, the iteration diverges under tall columns). */
    const double ir0 = 1.0 / (P->rho0 * P->rho0);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < P->n; ++i) {
        double acc[3] = {0, 0, 0};
        const double pV1 = clamp ? p[i] * ir0 : p[i] / (rho[i] * rho[i]);
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            const double dv[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            const double d = len3(dv);
            if (!(d > 0)) continue;
            if (clamp && d >= h) continue;
            const double inv = 1.0 / d;
            const double pV2 = clamp ? p[j] * ir0 : p[j] / (rho[j] * rho[j]);
            const double a = PI_D * pow(h, 6);
            const double s = -45 * pow(h - d, 2) / a;
            for (int e = 0; e < 3; ++e) acc[e] = acc[e] + (dv[e] * inv) * s * (pV1 + pV2) * m;
        }
        if (clamp) {
            walls_t w;
            near_walls(P, &pos[3 * i], &w);
            for (int mask = 1; mask < (1 << w.n); ++mask)
                for (int32_t t = 0; t < counts[i]; ++t) {
                    const int32_t j = list[(size_t)i * cap + t];
                    double dv[3], dpg;
                    if (!ghost(P, &w, mask, &pos[3 * i], &pos[3 * j], h, dv, &dpg)) continue;
                    const double d = len3(dv);
                    if (!(d > 0) || d >= h) continue;
                    const double inv = 1.0 / d;
                    /* the ghost continues the hydrostatic pressure across the face */
                    const double pV2 = (p[j] + dpg) * ir0;
                    const double a = PI_D * pow(h, 6);
                    const double sc = -45 * pow(h - d, 2) / a;
                    for (int e = 0; e < 3; ++e) acc[e] = acc[e] + (dv[e] * inv) * sc * (pV1 + pV2) * m;
                }
            for (int32_t tb = 0; tb < bnd_count(P, i); ++tb) {     /* boundary particles: p_i mirrored */
                const int32_t b = bnd_at(P, i, tb);
                const double dv[3] = {pos[3 * i] - P->bnd_pos[3 * b], pos[3 * i + 1] - P->bnd_pos[3 * b + 1],
                                      pos[3 * i + 2] - P->bnd_pos[3 * b + 2]};
                const double d = len3(dv);
                if (!(d > 0) || d >= h) continue;
                const double inv = 1.0 / d;
                const double a = PI_D * pow(h, 6);
                const double sc = -45 * pow(h - d, 2) / a;
                for (int e = 0; e < 3; ++e) acc[e] = acc[e] + (dv[e] * inv) * sc * pV1 * P->bnd_psi[b];
            }
        }
        for (int e = 0; e < 3; ++e) fp[3 * i + e] = acc[e] * (-rho[i]);
    }
}

void orc_boundary_reaction(const orc_params* P, const double* pos, const double* p, int32_t nb, const double* bpos,
                           const double* psi, double* out) {
    const double h = P->h, m = P->mass, ir0 = 1.0 / (P->rho0 * P->rho0);
#pragma omp parallel for schedule(static)
    for (int32_t b = 0; b < nb; ++b) {
        double F[3] = {0, 0, 0};
        for (int32_t i = 0; i < P->n; ++i) {
            const double dv[3] = {pos[3 * i] - bpos[3 * b], pos[3 * i + 1] - bpos[3 * b + 1],
                                  pos[3 * i + 2] - bpos[3 * b + 2]};
            const double d = len3(dv);
            if (!(d > 0) || d >= h) continue;
            const double g = 45 * pow(h - d, 2) / (PI_D * pow(h, 6));
            for (int e = 0; e < 3; ++e) F[e] -= m * psi[b] * p[i] * ir0 * g * dv[e] / d;
        }
        for (int e = 0; e < 3; ++e) out[3 * b + e] = F[e];
    }
}

void orc_pressure_force(const orc_params* P, const double* pos, const double* rho, const double* p,
                        const int32_t* counts, const int32_t* list, int32_t cap, double* fp) {
    pressure_forces(P, pos, rho, p, counts, list, cap, fp);
}

double orc_pci_delta(const orc_params* P) {
    const double h = P->h, m = P->mass, rho0 = P->rho0, dt = (double)P->dt;
    const double s = P->spacing > 0 ? P->spacing : cbrt(m / rho0);
    const double G = 45.0 / (PI_D * h * h * h * h);
    const int R = (int)ceil(h / s);
    double W1[3] = {0, 0, 0}, W2 = 0;
    for (int k = -R; k <= R; ++k)
        for (int j = -R; j <= R; ++j)
            for (int i = -R; i <= R; ++i) {
                if (!i && !j && !k) continue;
                const double r = s * sqrt((double)(i * i + j * j + k * k));
                if (r >= h) continue;
                const double g = G * (1.0 - r / h) * (1.0 - r / h);
                const double d[3] = {i * s / r, j * s / r, k * s / r};
                for (int e = 0; e < 3; ++e) W1[e] += -g * d[e];
                W2 += g * g;
            }
    const double beta = 2.0 * (m * dt / rho0) * (m * dt / rho0);
    return 1.0 / (beta * (W1[0] * W1[0] + W1[1] * W1[1] + W1[2] * W1[2] + W2));
}

/* Config profile: p_i = max(0, p_i + delta (rho*_i - rho0)) for every
 * particle with the prototype delta (orc_pci_delta). */
static void pressure_update_config(const orc_params* P, const double* rho, double* p) {
    const double delta = orc_pci_delta(P);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < P->n; ++i) {
        const double v = p[i] + delta * (rho[i] - P->rho0);
        p[i] = RND(P, v > 0 ? v : 0.0);
    }
}

/* PCISPH pressure increment (PciSphSystem_Kernel.cu:43-64): only compressed
 * particles change, p += (rho - rho0) / (beta (|sum gradW|^2 + sum |gradW|^2)). */
static void pressure_update(const orc_params* P, const double* pos, const double* rho, const int32_t* counts,
                            const int32_t* list, int32_t cap, double* p) {
    const double h = P->h, m = P->mass, rho0 = P->rho0;
    const double dt = (double)P->dt;
    const int clamp = P->profile == ORC_PROFILE_CONFIG;
    if (clamp) { pressure_update_config(P, rho, p); return; }
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < P->n; ++i) {
        if (!(rho[i] > rho0)) continue;
        const double beta = 2 * pow(m * dt / rho0, 2);
        double press = rho[i] - rho0;
        double W1[3] = {0, 0, 0}, W2 = 0;
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            const double dv[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            const double d = len3(dv);
            if (!(d > 0)) continue;
            if (clamp && d >= h) continue;
            const double inv = 1.0 / d;
            const double a = PI_D * pow(h, 6);
            const double s = -45 * pow(h - d, 2) / a;
            double dW[3];
            for (int e = 0; e < 3; ++e) dW[e] = (dv[e] * inv) * s;
            W2 += dW[0] * dW[0] + dW[1] * dW[1] + dW[2] * dW[2];
            for (int e = 0; e < 3; ++e) W1[e] = W1[e] + dW[e];
        }
        if (W2 > 0) {
            press = -press / (beta * (-(W1[0] * W1[0] + W1[1] * W1[1] + W1[2] * W1[2]) - W2));
            p[i] = RND(P, p[i] + press);
        }
    }
}

/* Penalty walls (config profile): a = K*depth - C*v_n along each axis on
 * which x lies outside the box faces (an uploaded state; the projection
 * below keeps stepped particles inside). */
static void wall_accel(const orc_params* P, const double* x, const double* v, double* a) {
    for (int e = 0; e < 3; ++e) {
        a[e] = 0.0;
        const float lo = P->box_min[e], hi = P->box_max[e];
        if (x[e] < lo) a[e] += P->wall_k * (lo - x[e]) - P->wall_c * v[e];
        if (x[e] > hi) a[e] += -P->wall_k * (x[e] - hi) - P->wall_c * v[e];
    }
}

/* collisionBox (BoxCollision_Kernel.cu:7-34) on (pos, vel_ap): the bounds
 * Max - r and Min + r are float expressions there. PCISPH in both profiles:
 * in the config profile it keeps every particle at least r from each face,
 * where its own ghost still pushes back (on or behind a face a particle
 * meets its ghost at distance 0, which exerts no force, and its density
 * error could not be corrected). Config WCSPH keeps the penalty walls its
 * scene states. */
static void box_project(const orc_params* P, double* x, double* v) {
    const float r = P->particle_radius;
    double pI[3] = {x[0], x[1], x[2]}, nI[3] = {0, 0, 0};
    for (int e = 0; e < 3; ++e) {
        const float hi = P->box_max[e] - r;
        if (x[e] >= hi) { pI[e] = hi; nI[e] = -1.0; }
    }
    for (int e = 0; e < 3; ++e) {
        const float lo = P->box_min[e] + r;
        if (x[e] <= lo) { pI[e] = lo; nI[e] = 1.0; }
    }
    const double ln = len3(nI);
    if (ln > 0) {
        for (int e = 0; e < 3; ++e) nI[e] = nI[e] / ln;
        const double vd = v[0] * nI[0] + v[1] * nI[1] + v[2] * nI[2];
        for (int e = 0; e < 3; ++e) { x[e] = pI[e]; v[e] = v[e] - (1 + 0.0) * vd * nI[e]; }
    }
}

/* ---- collision objects ------------------------------------------------------
 * Each object as its reference kernel executes, FP64 where the reference is
 * FP64 and float where it computes in float (float3 temporaries, powf):
 *   plane ..... src/Kernel/Collision/PlaneCollision/PlaneCollision_Kernel.cu:7-81
 *   sphere .... SphereCollision/SphereCollision_Kernel.cu:7-91 with the launch of
 *               SphereCollision.cu:9-16, which hands the kernel dt as its
 *               `container` and the container flag as its dt
 *   cylinder .. CylinderCollision/CylinderCollision_Kernel.cu:4-103
 *   mesh ...... MeshCollision/MeshCollision_Kernel.cu:14-137
 *   heights ... HeightField/{Linear,Gaussian,Periodic}/*HeightFieldCollision_Kernel.cu
 * A plane particle that did not move is left alone (the reference divides
 * by zero there). Squares the reference takes with powf are float products. */

static inline float fsqf(float a) { return a * a; }
static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline float dot3f(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* v -= (1 + r) (v.n) n, r float */
static void coll_reflect(double* v, const double* n, float r) {
    const double k = (double)(1.f + r) * dot3(v, n);
    for (int e = 0; e < 3; ++e) v[e] = v[e] - k * n[e];
}

static float coll_restitution(float elast, float dt, const double* x, const double* xc, const double* v) {
    const double lv = len3(v);
    if (lv > 0 && elast > 0) {
        const double d[3] = {x[0] - xc[0], x[1] - xc[1], x[2] - xc[2]};
        return (float)((double)elast * len3(d) / ((double)dt * lv));
    }
    return 0.f;
}

static int coll_plane(const orc_collider* o, float dt, const double* xo, double* x, double* v) {
    const float* q = o->v;
    const float* N = q + 12;
    float lo[3] = {100000.f, 100000.f, 100000.f}, hi[3] = {-100000.f, -100000.f, -100000.f};
    for (int c = 0; c < 4; ++c)
        for (int a = 0; a < 3; ++a) {
            if (lo[a] >= q[3 * c + a]) lo[a] = q[3 * c + a];
            if (hi[a] <= q[3 * c + a]) hi[a] = q[3 * c + a];
        }
    for (int a = 0; a < 3; ++a) {
        const float s = 1.f - N[a];
        const double xa = x[a] * (double)s;
        if (!(xa <= (double)(hi[a] * s) && xa >= (double)(lo[a] * s))) return 0;
    }
    float p1[3], ao[3], dir[3];
    for (int a = 0; a < 3; ++a) {
        p1[a] = (float)(x[a] - (double)q[a]);
        ao[a] = (float)((double)q[a] - xo[a]);
        dir[a] = (float)(x[a] - xo[a]);
    }
    if (!(dot3f(p1, N) <= 0.f)) return 0;
    const float ao_n = dot3f(ao, N);
    const float dn = sqrtf(dot3f(dir, dir));
    if (!(dn > 0.f)) return 0;
    for (int a = 0; a < 3; ++a) dir[a] = dir[a] / dn;
    const float t = ao_n / dot3f(dir, N);
    double xc[3], n[3];
    for (int a = 0; a < 3; ++a) xc[a] = xo[a] + (double)(t * dir[a]);
    const float r = coll_restitution(o->elast, dt, x, xc, v);
    const double nw[3] = {N[0], N[1], N[2]};
    const double ln = len3(nw);
    for (int a = 0; a < 3; ++a) n[a] = nw[a] / ln;
    for (int a = 0; a < 3; ++a) x[a] = xc[a];
    coll_reflect(v, n, r);
    return 1;
}

static int coll_sphere(const orc_collider* o, float dt, double* x, double* v) {
    const int inside = dt != 0.f;
    const float dt_k = o->container ? 1.f : 0.f;
    const double c[3] = {o->v[0], o->v[1], o->v[2]};
    const double R = (double)o->v[3];
    const double op[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
    const double d = len3(op);
    double xc[3], n[3];
    if ((inside && d == R) || (!inside && d == R)) {
        const double rd = 1.0f / d;          /* double3.h operator/: times the reciprocal */
        for (int a = 0; a < 3; ++a) { xc[a] = x[a]; n[a] = -op[a] * rd; }
    } else if (inside && d > R) {
        const double rd = 1.0f / d;
        for (int a = 0; a < 3; ++a) xc[a] = c[a] + (op[a] * rd) * R;
        const double w[3] = {c[0] - xc[0], c[1] - xc[1], c[2] - xc[2]};
        const double rl = 1.0f / len3(w);
        for (int a = 0; a < 3; ++a) n[a] = w[a] * rl;
    } else {
        return 0;
    }
    const float r = coll_restitution(o->elast, dt_k, x, xc, v);
    const double ln = len3(n);
    for (int a = 0; a < 3; ++a) n[a] = n[a] / ln;
    for (int a = 0; a < 3; ++a) x[a] = xc[a];
    coll_reflect(v, n, r);
    return 1;
}

static double fdist3(const double* a, const double* b) {
    return (double)sqrtf(fsqf((float)(a[0] - b[0])) + fsqf((float)(a[1] - b[1])) + fsqf((float)(a[2] - b[2])));
}

static int coll_cylinder(const orc_collider* o, float dt, double* x, double* v) {
    const float* ce = o->v;
    const float* di = o->v + 3;
    const float rb = o->v[6], l = o->v[7];
    double p1[3], p2[3], C[3], cd[3], xc[3] = {x[0], x[1], x[2]}, n[3];
    for (int a = 0; a < 3; ++a) {
        p1[a] = (double)(ce[a] + di[a] * (l / 2));
        p2[a] = (double)(ce[a] - di[a] * (l / 2));
        cd[a] = (double)ce[a];
    }
    C[0] = (double)ce[0] + x[0] * (double)di[0];
    C[1] = (double)ce[1] + x[1] * (double)di[1];
    C[2] = (double)ce[2] + x[2] * (double)di[0];    /* the reference's z takes direction.x */
    const double margin = (double)rb - 0.04;
    const float dl = sqrtf(fsqf(di[0]) + fsqf(di[1]) + fsqf(di[2]));
    const double w[3] = {C[0] - x[0], C[1] - x[1], C[2] - x[2]};
    const double lw = len3(w);
    if (fdist3(cd, C) >= (double)(l / 2)) {
        const int low = fdist3(p1, C) > fdist3(p2, C);   /* nearer the P2 end */
        const double* pe = low ? p2 : p1;
        double u[3];
        for (int a = 0; a < 3; ++a) u[a] = low ? w[a] / lw : -w[a] / lw;
        for (int a = 0; a < 3; ++a)
            if (di[a] != 0.f) xc[a] = pe[a];
        if (lw >= (double)rb)
            for (int a = 0; a < 3; ++a)
                if (di[a] == 0.f) xc[a] = low ? C[a] - margin * u[a] : C[a] + margin * u[a];
        for (int a = 0; a < 3; ++a) n[a] = (double)(low ? di[a] : -di[a]) / (double)dl;
    } else {
        if (!(fdist3(C, x) >= (double)rb)) return 0;
        for (int a = 0; a < 3; ++a) {
            n[a] = -w[a] / lw;
            xc[a] = C[a] + margin * n[a] * (double)(1.f - di[a]);
        }
    }
    float r = 0.f;
    const double lv = len3(v);
    if (lv > 0 && dt > 0.f) {
        const double d[3] = {x[0] - xc[0], x[1] - xc[1], x[2] - xc[2]};
        r = (float)((double)0.3f * len3(d) / ((double)dt * lv));
    }
    for (int a = 0; a < 3; ++a) x[a] = xc[a];
    coll_reflect(v, n, r);
    return 1;
}

static int in_triangle(const float* A, const float* B, const float* Cc, const float* P) {
    float u[3], w[3], p[3];
    for (int a = 0; a < 3; ++a) { u[a] = B[a] - A[a]; w[a] = Cc[a] - A[a]; p[a] = P[a] - A[a]; }
    const float uu = dot3f(u, u), uw = dot3f(u, w), ww = dot3f(w, w), pu = dot3f(p, u), pw = dot3f(p, w);
    const float D = uw * uw - uu * ww;
    const float s = (uw * pw - ww * pu) / D;
    if (s < 0.f || s > 1.f) return 0;
    const float t = (uw * pu - uu * pw) / D;
    if (t < 0.f || (s + t) > 1.f) return 0;
    return 1;
}

static int coll_mesh(const orc_collider* o, const double* xo, double* x, double* v) {
    double best = 10000000, xb[3] = {x[0], x[1], x[2]}, nb[3] = {0, 0, 0};
    int found = 0;
    for (int32_t f = 0; f < o->count; ++f) {
        const float* A = o->faces + 12 * (size_t)f;
        const float* N = A + 9;
        const double Nd[3] = {N[0], N[1], N[2]};
        const double p1[3] = {x[0] - A[0], x[1] - A[1], x[2] - A[2]};
        const double d1 = dot3(p1, Nd);
        if (!(d1 <= 0)) continue;
        const double dir0[3] = {xo[0] - x[0], xo[1] - x[1], xo[2] - x[2]};
        const double dn = len3(dir0);
        double xc[3];
        if (d1 == 0 || dn <= 0 || d1 == -1) {
            for (int a = 0; a < 3; ++a) xc[a] = x[a];
        } else {
            const double ao[3] = {A[0] - x[0], A[1] - x[1], A[2] - x[2]};
            const double ao_n = dot3(ao, Nd);
            const double dir[3] = {dir0[0] / dn, dir0[1] / dn, dir0[2] / dn};
            const double t = ao_n / dot3(dir, Nd);
            for (int a = 0; a < 3; ++a) xc[a] = xo[a] + t * dir[a];
            const float pf[3] = {(float)xc[0], (float)xc[1], (float)xc[2]};
            if (!in_triangle(A, A + 3, A + 6, pf)) continue;
        }
        const double dist = fdist3(x, xc);
        if (dist <= best) {
            best = dist;
            for (int a = 0; a < 3; ++a) { xb[a] = xc[a]; nb[a] = Nd[a]; }
            found = 1;
        }
    }
    if (!found) return 0;
    for (int a = 0; a < 3; ++a) x[a] = xb[a];
    coll_reflect(v, nb, 0.f);
    return 1;
}

static double height_of(const orc_collider* o, double x, double z) {
    double y = 0;
    for (int32_t i = 0; i < o->count; ++i) {
        const double* c = o->terms + 6 * (size_t)i;
        const int kind = (int)c[0];
        if (kind == 1) y += c[1] * x + c[2] * z;
        else if (kind == 2)
            y += c[1] * exp(-((double)fsqf((float)(x - c[2])) / (2 * c[4] * c[4]) +
                              (double)fsqf((float)(z - c[3])) / (2 * c[5] * c[5])));
        else y += c[1] * cos(c[2] * (x * cos(c[3]) + z * sin(c[3])) + c[4]);
    }
    return y;
}

static int coll_height(const orc_collider* o, float dt, double* x, double* v) {
    const float* q = o->v;
    if (!(x[0] >= (double)q[0] && x[2] >= (double)q[2] && x[0] <= (double)q[3] && x[2] <= (double)q[5])) return 0;
    const double y = height_of(o, x[0], x[2]) + (double)q[1];
    if (!(y >= x[1])) return 0;
    const double xc[3] = {x[0], y, x[2]};
    const float r = coll_restitution(o->elast, dt, x, xc, v);
    const double d = 0.01;
    const double dpx = (height_of(o, xc[0] + d, xc[2]) - height_of(o, xc[0] - d, xc[2])) / (2 * d);
    const double dpz = (height_of(o, xc[0], xc[2] + d) - height_of(o, xc[0], xc[2] - d)) / (2 * d);
    const double nn = sqrt(dpx * dpx + 1.0 + dpz * dpz);
    double n[3] = {-dpx / nn, 1.0 / nn, -dpz / nn};
    const double ln = len3(n);
    for (int a = 0; a < 3; ++a) n[a] = n[a] / ln;
    x[1] = y;
    coll_reflect(v, n, r);
    return 1;
}

static int collide_one(const orc_collider* o, float dt, const double* xo, double* x, double* v) {
    switch (o->type) {
        case 1: return coll_plane(o, dt, xo, x, v);
        case 2: return coll_sphere(o, dt, x, v);
        case 3: return coll_cylinder(o, dt, x, v);
        case 4: return coll_mesh(o, xo, x, v);
        case 5: return coll_height(o, dt, x, v);
        default: return 0;
    }
}

int32_t orc_collide(const orc_collider* o, int32_t n, const double* old_pos, double* pos, double* vel, float dt) {
    int32_t hits = 0;
#pragma omp parallel for schedule(static) reduction(+ : hits)
    for (int32_t i = 0; i < n; ++i)
        hits += collide_one(o, dt, old_pos ? &old_pos[3 * i] : &pos[3 * i], &pos[3 * i], &vel[3 * i]);
    return hits;
}

/* Every object of P's list on one particle, after the box. */
static void collide_all(const orc_params* P, const double* xo, double* x, double* v) {
    for (int32_t k = 0; k < P->n_coll; ++k) collide_one(&P->coll[k], P->dt, xo, x, v);
}

/* ---- steps ---------------------------------------------------------------- */

static int32_t* build_lists(const orc_params* P, const double* pos, int32_t* counts, int32_t* cap_out, orc_stats* st) {
    orc_neighbors(P, pos, 0, counts, NULL);
    int32_t cap = 1;
    int64_t tot = 0;
    for (int32_t i = 0; i < P->n; ++i) { cap = counts[i] > cap ? counts[i] : cap; tot += counts[i]; }
    int32_t* list = (int32_t*)malloc(sizeof(int32_t) * (size_t)P->n * cap);
    orc_neighbors(P, pos, cap, counts, list);
    if (st) {
        st->nbr_total = tot;
        st->nbr_max = cap;
        uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)P->n);
        orc_cell_keys(P->n, pos, P->grid_min, P->cell, P->dims, keys, &st->clamped);
        free(keys);
    }
    *cap_out = cap;
    return list;
}

static int step_wcsph(const orc_params* P, orc_state* S, orc_stats* st, double* rho_x, double* f_np, int32_t* nbr_counts) {
    const int32_t n = P->n;
    const int ref = P->profile == ORC_PROFILE_REF;
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t cap = 0;
    int32_t* list = build_lists(P, S->pos, counts, &cap, st);
    /* boundary particles: lists at the start positions, like the fluid's */
    orc_params Qb;
    int32_t *bnd_counts = NULL, *bnd_lists = NULL;
    if (P->n_bnd > 0) {
        Qb = *P;
        build_bnd_lists(P, S->pos, &bnd_counts, &bnd_lists, &Qb.bnd_cap);
        Qb.bnd_counts = bnd_counts;
        Qb.bnd_lists = bnd_lists;
        P = &Qb;
    }
    double* rho = S->rho;
    double* p = S->p;
    double* fnp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    double* fp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    if (ref) {
        /* densityEvaluation (SphKernel.cu:9-27) */
        const double h = P->h, m = P->mass;
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int32_t t = 0; t < counts[i]; ++t) {
                const int32_t j = list[(size_t)i * cap + t];
                const double dv[3] = {S->pos[3 * i] - S->pos[3 * j], S->pos[3 * i + 1] - S->pos[3 * j + 1],
                                      S->pos[3 * i + 2] - S->pos[3 * j + 2]};
                const double d = len3(dv);
                const double a = 64 * PI_D * pow(h, 9);
                const double m_k = 315 / a;
                const double b = pow((h * h) - (d * d), 3);
                s += b * m_k * m;
            }
            rho[i] = RND(P, s);
            p[i] = RND(P, P->k * (rho[i] - P->rho0));
        }
    } else {
        orc_density(P, S->pos, counts, list, cap, 1, rho);
        const double B = P->k * P->rho0 / 7.0;
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) p[i] = RND(P, B * (pow(rho[i] / P->rho0, 7) - 1.0));
    }
    if (rho_x) memcpy(rho_x, rho, sizeof(double) * (size_t)n);
    nonpressure_forces(P, S->pos, S->vel, rho, counts, list, cap, fnp);
    pressure_forces(P, S->pos, rho, p, counts, list, cap, fp);
    if (f_np) memcpy(f_np, fnp, sizeof(double) * 3 * (size_t)n);
    const double dt = (double)P->dt;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        double* x = &S->pos[3 * i];
        double* vap = &S->vel_ap[3 * i];
        double aw[3] = {0, 0, 0};
        if (!ref) wall_accel(P, x, vap, aw);
        const double vav[3] = {vap[0], vap[1], vap[2]};
        const double xo[3] = {x[0], x[1], x[2]};
        const double inv = 1.0 / rho[i];
        for (int e = 0; e < 3; ++e) {
            /* internalForces accumulates visc + surf + press, then the force
             * kernel adds rho*g: F = ((fv + fs) + fp) + g */
            const double F = fnp[3 * i + e] + fp[3 * i + e];
            vap[e] = RND(P, vap[e] + (F * inv + aw[e]) * dt);
            x[e] = RND(P, x[e] + vap[e] * dt);
        }
        if (ref) box_project(P, x, vap);   /* config WCSPH: penalty walls only */
        collide_all(P, xo, x, vap);
        for (int e = 0; e < 3; ++e) {
            x[e] = RND(P, x[e]);
            vap[e] = RND(P, vap[e]);
            S->vel[3 * i + e] = RND(P, (vav[e] + vap[e]) / 2);
        }
    }
    if (nbr_counts) memcpy(nbr_counts, counts, sizeof(int32_t) * (size_t)n);
    if (st) { st->iters = 0; st->converged = 1; }
    free(counts); free(list); free(fnp); free(fp);
    free(bnd_counts);
    free(bnd_lists);
    return 0;
}

/* Moving boundary (P->bnd_vel set): the fluid's reaction F_b on every
 * boundary particle at pressures p, over the fluid's boundary lists at the
 * start positions (in fluid-particle order, so the sums are deterministic),
 * and the boundary prediction x*_b = x_b + dt (v_b + dt (F_b + f_b) / m_b).
 * F_b = -sum_i m psi_b (p_i / rho0^2) 45 (h - d)^2 / (pi h^6) (x_i - x_b) / d,
 * the reaction to the mirrored-pressure force (as orc_boundary_reaction). */
static void move_boundary(const orc_params* P, const double* pos, const double* p, double* F, double* pred) {
    const int32_t nb = P->n_bnd;
    const double h = P->h, m = P->mass, ir0 = 1.0 / (P->rho0 * P->rho0), dt = (double)P->dt;
    memset(F, 0, sizeof(double) * 3 * (size_t)nb);
    for (int32_t i = 0; i < P->n; ++i) {
        for (int32_t t = 0; t < bnd_count(P, i); ++t) {
            const int32_t b = bnd_at(P, i, t);
            const double dv[3] = {pos[3 * i] - P->bnd_pos[3 * b], pos[3 * i + 1] - P->bnd_pos[3 * b + 1],
                                  pos[3 * i + 2] - P->bnd_pos[3 * b + 2]};
            const double d = len3(dv);
            if (!(d > 0) || d >= h) continue;
            const double g = 45 * pow(h - d, 2) / (PI_D * pow(h, 6));
            for (int e = 0; e < 3; ++e) F[3 * b + e] -= m * P->bnd_psi[b] * p[i] * ir0 * g * dv[e] / d;
        }
    }
    for (int32_t b = 0; b < nb; ++b)
        for (int e = 0; e < 3; ++e) {
            const double v = P->bnd_vel[3 * b + e] + dt * (F[3 * b + e] + P->bnd_fext[3 * b + e]) * P->bnd_inv_mass;
            pred[3 * b + e] = RND(P, P->bnd_pos[3 * b + e] + dt * RND(P, v));
        }
}

static int step_pcisph(const orc_params* P, orc_state* S, orc_stats* st, double* rho_x, double* f_np, int32_t* nbr_counts) {
    if (st) memset(st, 0, sizeof(*st));
    const int32_t n = P->n;
    const int ref = P->profile == ORC_PROFILE_REF;
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t cap = 0;
    int32_t* list = build_lists(P, S->pos, counts, &cap, st);
    /* boundary particles: lists at the start positions, like the fluid's */
    orc_params Qb;
    int32_t *bnd_counts = NULL, *bnd_lists = NULL;
    if (P->n_bnd > 0) {
        Qb = *P;
        build_bnd_lists(P, S->pos, &bnd_counts, &bnd_lists, &Qb.bnd_cap);
        Qb.bnd_counts = bnd_counts;
        Qb.bnd_lists = bnd_lists;
        P = &Qb;
    }
    const size_t n3 = 3 * (size_t)n;
    double* rho = (double*)malloc(sizeof(double) * (size_t)n);
    double* fnp = (double*)malloc(sizeof(double) * n3);
    double* fp = (double*)calloc(n3, sizeof(double));
    double* xs = (double*)malloc(sizeof(double) * n3);
    double* vs = (double*)malloc(sizeof(double) * n3);
    double* aw = (double*)calloc(n3, sizeof(double));
    double* p = S->p;

    orc_density(P, S->pos, counts, list, cap, !ref, rho);
    if (rho_x) memcpy(rho_x, rho, sizeof(double) * (size_t)n);
    nonpressure_forces(P, S->pos, S->vel, rho, counts, list, cap, fnp);
    if (f_np) memcpy(f_np, fnp, sizeof(double) * n3);
    if (!ref) {
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) wall_accel(P, &S->pos[3 * i], &S->vel_ap[3 * i], &aw[3 * i]);
    }
    if (ref || !P->warm_start) memset(p, 0, sizeof(double) * (size_t)n);
    else pressure_forces(P, S->pos, rho, p, counts, list, cap, fp);   /* warm start: f_p of the initial guess at x */
    /* moving boundary: the density passes see the predicted boundary */
    const int moving = !ref && P->n_bnd > 0 && P->bnd_vel && P->bnd_pred && P->bnd_force;
    orc_params Qm;
    const orc_params* Pd = P;
    if (moving) {
        move_boundary(P, S->pos, p, P->bnd_force, P->bnd_pred);
        Qm = *P;
        Qm.bnd_pos = P->bnd_pred;
        Pd = &Qm;
    }

    const double dt = (double)P->dt;
    const int min_it = ref ? 3 : P->min_iters, max_it = ref ? 3 : P->max_iters;
    int k = 0, converged = 0;
    for (;;) {
        /* predict (integrateSPH_LeapFrog_Forces on the saved state, SphKernel.cu:95-108) */
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            const double inv = 1.0 / rho[i];
            for (int e = 0; e < 3; ++e) {
                const double F = fnp[3 * i + e] + fp[3 * i + e];
                vs[3 * i + e] = RND(P, S->vel_ap[3 * i + e] + (F * inv + aw[3 * i + e]) * dt);
                xs[3 * i + e] = RND(P, S->pos[3 * i + e] + vs[3 * i + e] * dt);
            }
        }
        if (k >= max_it) break;
        double* rs = (double*)malloc(sizeof(double) * (size_t)n);
        orc_density(Pd, xs, counts, list, cap, !ref, rs);
        double err = 0.0;
        for (int32_t i = 0; i < n; ++i) {
            const double e = (rs[i] - P->rho0) / P->rho0;
            err = e > err ? e : err;
        }
        if (st && k <= ORC_MAX_ITERS) st->err[k] = err;
        memcpy(rho, rs, sizeof(double) * (size_t)n);
        free(rs);
        if (!ref && k >= min_it && err <= P->eta) { converged = 1; break; }
        pressure_update(P, xs, rho, counts, list, cap, p);
        /* reference: force at the predicted positions (PciSphSystem.cu:53-56);
         * config: at the step's start positions, so that the corrector is a
         * linear iteration in p (at x*, x* = x + dt^2 a(x*) is itself a
         * fixed-point iteration that diverges once p dt^2/h^2 grows, as it
         * does under a 0.64 m column) */
        pressure_forces(P, ref ? xs : S->pos, rho, p, counts, list, cap, fp);
        if (moving) move_boundary(P, S->pos, p, P->bnd_force, P->bnd_pred);
        k++;
    }
    /* config: XSPH smoothing of the committed velocity (Monaghan 1989),
     * v_i + xsph sum_j (m/rho0) W_ij (v_j - v_i) at x*; positions stay */
    if (!ref && P->xsph > 0) {
        const double h = P->h, kw = P->xsph * 315.0 * P->mass / (64.0 * PI_D * h * h * h) / P->rho0;
        double* vx = (double*)malloc(sizeof(double) * n3);
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            double dv[3] = {0, 0, 0};
            for (int32_t t = 0; t < counts[i]; ++t) {
                const int32_t j = list[(size_t)i * cap + t];
                const double d[3] = {xs[3 * i] - xs[3 * j], xs[3 * i + 1] - xs[3 * j + 1], xs[3 * i + 2] - xs[3 * j + 2]};
                const double q = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / (h * h);
                if (q >= 1.0) continue;
                const double w = (1 - q) * (1 - q) * (1 - q);
                for (int e = 0; e < 3; ++e) dv[e] += w * (vs[3 * j + e] - vs[3 * i + e]);
            }
            for (int e = 0; e < 3; ++e) vx[3 * i + e] = RND(P, vs[3 * i + e] + kw * dv[e]);
        }
        memcpy(vs, vx, sizeof(double) * n3);
        free(vx);
    }
    /* commit the last prediction; walls; velocity interpolation (SphKernel.cu:128-135) */
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        double* x = &S->pos[3 * i];
        double* vap = &S->vel_ap[3 * i];
        const double vav[3] = {vap[0], vap[1], vap[2]};
        const double xo[3] = {x[0], x[1], x[2]};
        for (int e = 0; e < 3; ++e) { x[e] = xs[3 * i + e]; vap[e] = vs[3 * i + e]; }
        box_project(P, x, vap);
        collide_all(P, xo, x, vap);
        for (int e = 0; e < 3; ++e) {
            x[e] = RND(P, x[e]);
            vap[e] = RND(P, vap[e]);
            S->vel[3 * i + e] = RND(P, (vav[e] + vap[e]) / 2);
        }
        S->rho[i] = rho[i];
    }
    if (nbr_counts) memcpy(nbr_counts, counts, sizeof(int32_t) * (size_t)n);
    if (st) { st->iters = k; st->converged = ref ? 1 : converged; }
    free(counts); free(list); free(rho); free(fnp); free(fp); free(xs); free(vs); free(aw);
    free(bnd_counts);
    free(bnd_lists);
    return 0;
}

/* Inputs of the learned pressure warm start (config-profile PCISPH) at the
 * step's start positions, seven per particle. The reference has no
 * counterpart: every reference step starts from p = 0
 * (PciSphSystem_Kernel.cu:131). Sums run over the neighbour list (self
 * included, pairs with r >= h dropped); rho is the density at x with the
 * wall ghosts and boundary particles, as the step computes it.
 *   f0 neighbour count / 32
 *   f1 advected density deviation (rho - dt rho div v - rho0) / rho0 * 100
 *   f2 div v * dt * 100, div v = (1/rho0) sum_j m (v_j - v_i) . gradW_ij
 *   f3 previous pressure / p_scale
 *   f4 distance to the nearest box face / h, in [0, 1]
 *   f5 |sum_j m gradW_ij| * h / rho0
 *   f6 sum_j W_ij p_j / sum_j W_ij / p_scale (poly6 weights, 0 if none)
 * with gradW the spiky gradient -45/(pi h^6) (h - r)^2 x_ij/r and p_scale
 * = rho0 |g| 0.1 m (|g| = 9.81 when gravity is zero). */
void orc_features(const orc_params* P, const double* pos, const double* vel, const double* p_prev, double* out) {
    const int32_t n = P->n;
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t cap = 0;
    int32_t* list = build_lists(P, pos, counts, &cap, NULL);
    orc_params Qb;
    int32_t *bnd_counts = NULL, *bnd_lists = NULL;
    if (P->n_bnd > 0) {
        Qb = *P;
        build_bnd_lists(P, pos, &bnd_counts, &bnd_lists, &Qb.bnd_cap);
        Qb.bnd_counts = bnd_counts;
        Qb.bnd_lists = bnd_lists;
        P = &Qb;
    }
    double* rho = (double*)malloc(sizeof(double) * (size_t)n);
    orc_density(P, pos, counts, list, cap, 1, rho);
    const double h = P->h, m = P->mass, rho0 = P->rho0, dt = (double)P->dt;
    const double G = 45.0 / (PI_D * pow(h, 6));
    const double g = sqrt((double)P->gravity[0] * P->gravity[0] + (double)P->gravity[1] * P->gravity[1] +
                          (double)P->gravity[2] * P->gravity[2]);
    const double p_scale = rho0 * (g > 0 ? g : 9.81) * 0.1;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        const double* xi = &pos[3 * i];
        double div = 0.0, gr[3] = {0, 0, 0}, wp = 0.0, ws = 0.0;
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            const double d[3] = {xi[0] - pos[3 * j], xi[1] - pos[3 * j + 1], xi[2] - pos[3 * j + 2]};
            const double r = len3(d);
            if (r >= h) continue;
            const double w = (h * h - r * r) / (h * h);
            wp += w * w * w * p_prev[j];
            ws += w * w * w;
            if (r > 0) {
                const double gw = -G * (h - r) * (h - r) / r;     /* gradW_ij = gw * d */
                for (int e = 0; e < 3; ++e) {
                    div += m * (vel[3 * j + e] - vel[3 * i + e]) * gw * d[e];
                    gr[e] += m * gw * d[e];
                }
            }
        }
        div /= rho0;
        double dwall = h;
        for (int e = 0; e < 3; ++e) {
            const double lo = xi[e] - (double)P->box_min[e], hi = (double)P->box_max[e] - xi[e];
            dwall = lo < dwall ? lo : dwall;
            dwall = hi < dwall ? hi : dwall;
        }
        double* f = &out[7 * (size_t)i];
        f[0] = counts[i] / 32.0;
        f[1] = (rho[i] - dt * rho[i] * div - rho0) / rho0 * 100.0;
        f[2] = div * dt * 100.0;
        f[3] = p_prev[i] / p_scale;
        f[4] = (dwall > 0 ? dwall : 0.0) / h;
        f[5] = len3(gr) * h / rho0;
        f[6] = ws > 0 ? wp / ws / p_scale : 0.0;
    }
    free(counts); free(list); free(rho); free(bnd_counts); free(bnd_lists);
}

int orc_presolve(const orc_params* P, orc_state* S, int32_t iters, orc_stats* st) {
    /* The state is saved and restored around one warm-started step with
     * exactly `iters` corrections; only the pressure is kept. */
    orc_params Q = *P;
    Q.min_iters = Q.max_iters = iters;
    Q.eta = 0.0;
    Q.warm_start = 1;
    const size_t n3 = 3 * (size_t)P->n;
    double* save = (double*)malloc(sizeof(double) * (3 * n3 + (size_t)P->n));
    memcpy(save, S->pos, sizeof(double) * n3);
    memcpy(save + n3, S->vel, sizeof(double) * n3);
    memcpy(save + 2 * n3, S->vel_ap, sizeof(double) * n3);
    memcpy(save + 3 * n3, S->rho, sizeof(double) * P->n);
    const int rc = step_pcisph(&Q, S, st, NULL, NULL, NULL);
    memcpy(S->pos, save, sizeof(double) * n3);
    memcpy(S->vel, save + n3, sizeof(double) * n3);
    memcpy(S->vel_ap, save + 2 * n3, sizeof(double) * n3);
    memcpy(S->rho, save + 3 * n3, sizeof(double) * P->n);
    free(save);
    return rc;
}

/* ---- DEM (CudaSystem::update, CudaSystem.cpp:207-224) ----------------------
 * Forces start at zero plus the constant force m g (evaluate_force_constante,
 * ForceExt_Constante.cu:15-23: (dir amp) in float times the mass), then the
 * pair forces over the neighbour list on the step's start state, then
 * explicit Euler and the box. Reference profile: collideParticle
 * (CudaParticle_Kernel.cu:10-36) as it executes -- the spring term alone,
 * see dem_pair_ref -- with the interaction radius as the sphere radius, as
 * interactionSystem passes it (CudaSystem.cpp:244), and
 * integrateEuler (ParticleKernel.cu:12-20): x += v_old dt. Config profile
 * (the scene text's linear spring-dashpot): on an overlap delta = 2r - d > 0
 * of two particle_radius spheres, F_A = (-k_n delta + c_n (v_B - v_A).n) n
 * with n the unit vector from A to B; semi-implicit Euler, x += v_new dt. */
static void dem_pair_ref(const orc_params* P, const double* xa, const double* xb, const double* va, const double* vb,
                         double* f) {
    const double rel[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
    const double dist = sqrt((rel[0] * rel[0] + rel[1] * rel[1]) + rel[2] * rel[2]);
    if (!(dist > 0)) return;
    const float R = (float)(P->h + P->h);
    if (!(dist < R * 2.0f)) return;
    const double inv = 1.0 / dist;
    const double nrm[3] = {rel[0] * inv, rel[1] * inv, rel[2] * inv};
    (void)va; (void)vb;
    /* force = -spring (collideDist - dist) norm (CudaParticle_Kernel.cu:28).
     * The dashpot, shear and attraction lines (:30-34) are `force += ...`,
     * and the reference's double3 operator+= (double3.h:115-117) takes its
     * left operand by const reference and only returns the sum: those terms
     * never reach the force. */
    for (int e = 0; e < 3; ++e) f[e] = f[e] + (-P->dem_spring * ((double)R - dist) * nrm[e]);
}

static void dem_pair_config(const orc_params* P, const double* xa, const double* xb, const double* va,
                            const double* vb, double* f) {
    const double rel[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
    const double dist = sqrt(rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2]);
    const double delta = 2.0 * (double)P->particle_radius - dist;
    if (!(dist > 0) || !(delta > 0)) return;
    const double nrm[3] = {rel[0] / dist, rel[1] / dist, rel[2] / dist};
    const double vn = (vb[0] - va[0]) * nrm[0] + (vb[1] - va[1]) * nrm[1] + (vb[2] - va[2]) * nrm[2];
    const double s = -P->dem_spring * delta + P->dem_damping * vn;
    for (int e = 0; e < 3; ++e) f[e] += s * nrm[e];
}

static int step_dem(const orc_params* P, orc_state* S, orc_stats* st, double* f_out, int32_t* nbr_counts) {
    const int32_t n = P->n;
    const int ref = P->profile == ORC_PROFILE_REF;
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t cap = 0;
    int32_t* list = build_lists(P, S->pos, counts, &cap, st);
    double* f = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    const double dt = (double)P->dt;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        double* fi = &f[3 * (size_t)i];
        for (int e = 0; e < 3; ++e) fi[e] = 0.0 + (double)P->gravity[e] * P->mass;
        if (P->dem_ext)
            for (int e = 0; e < 3; ++e) fi[e] += P->dem_ext[3 * (size_t)i + e];
        for (int32_t t = 0; t < counts[i]; ++t) {
            const int32_t j = list[(size_t)i * cap + t];
            if (ref) dem_pair_ref(P, &S->pos[3 * i], &S->pos[3 * j], &S->vel[3 * i], &S->vel[3 * j], fi);
            else dem_pair_config(P, &S->pos[3 * i], &S->pos[3 * j], &S->vel[3 * i], &S->vel[3 * j], fi);
        }
    }
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        double* x = &S->pos[3 * i];
        double* v = &S->vel[3 * i];
        const double v0[3] = {v[0], v[1], v[2]};
        const double xo[3] = {x[0], x[1], x[2]};
        for (int e = 0; e < 3; ++e) {
            v[e] = RND(P, v[e] + (f[3 * i + e] / P->mass) * dt);
            x[e] = RND(P, x[e] + (ref ? v0[e] : v[e]) * dt);
        }
        box_project(P, x, v);    /* collisionBox on (pos, vel), CudaSystem::collide */
        collide_all(P, xo, x, v);
        for (int e = 0; e < 3; ++e) {
            x[e] = RND(P, x[e]);
            v[e] = RND(P, v[e]);
            S->vel_ap[3 * i + e] = v[e];
        }
    }
    if (f_out) for (size_t k = 0; k < 3 * (size_t)n; ++k) f_out[k] = RND(P, f[k]);
    if (nbr_counts) memcpy(nbr_counts, counts, sizeof(int32_t) * (size_t)n);
    if (st) { st->iters = 0; st->converged = 1; }
    free(counts); free(list); free(f);
    return 0;
}

int orc_step(const orc_params* P, orc_state* S, orc_stats* st, double* rho_x, double* f_np, int32_t* nbr_counts) {
    if (st) memset(st, 0, sizeof(*st));
    if (P->n <= 0) return 0;
    if (P->method == ORC_DEM) return step_dem(P, S, st, f_np, nbr_counts);
    if (P->method == ORC_PCISPH) return step_pcisph(P, S, st, rho_x, f_np, nbr_counts);
    return step_wcsph(P, S, st, rho_x, f_np, nbr_counts);
}

/* ---- iso field and marching cubes ------------------------------------------
 * Iso field, reference profile: evaluateIso_Kernel (UniformGridKernel.cu:
 * 98-138) -- the node's particle-grid cell (I, J, K) = floor((x - Min) /
 * sizeCell), floor(1/scale) rings of cells around it, and for each particle
 * with d = length(x - x_j) <= r = h/scale the float term
 * (1/powf(r,6)) * powf(r*r - d*d, 3) added to a double sum. Config profile:
 * the colour field sum_j (m/rho_j) 315/(64 pi h^9) (h^2 - d^2)^3 over the
 * adjacent cells. Cells are walked x outer, z inner, particles within a cell
 * in increasing id (the GPU's sorted order). */
void orc_iso_field(const orc_params* P, const double* pos, const double* rho, const orc_iso_grid* g, double* iso) {
    const int32_t n = P->n;
    const uint32_t ncells = (uint32_t)P->dims[0] * (uint32_t)P->dims[1] * (uint32_t)P->dims[2];
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* start = (int32_t*)malloc(sizeof(int32_t) * ((size_t)ncells + 1));
    orc_cell_keys(n, pos, P->grid_min, P->cell, P->dims, keys, NULL);
    sort_by_key(n, keys, ncells, perm, start);
    const int ref = P->profile == ORC_PROFILE_REF;
    const double h = P->h;
    const double r = ref ? h / g->scale : h;
    const int ring = ref ? (int)floor(1.0 / g->scale) : 1;
    const double kc = 315.0 * P->mass / (64.0 * PI_D * h * h * h);
    const int64_t nn = (int64_t)g->dims[0] * g->dims[1] * g->dims[2];
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t node = 0; node < nn; ++node) {
        const int ix = (int)(node % g->dims[0]), iy = (int)((node / g->dims[0]) % g->dims[1]);
        const int iz = (int)(node / ((int64_t)g->dims[0] * g->dims[1]));
        const double px = g->origin[0] + ix * g->spacing[0];
        const double py = g->origin[1] + iy * g->spacing[1];
        const double pz = g->origin[2] + iz * g->spacing[2];
        const int I = (int)floor((px - (double)P->grid_min[0]) / (double)P->cell);
        const int J = (int)floor((py - (double)P->grid_min[1]) / (double)P->cell);
        const int K = (int)floor((pz - (double)P->grid_min[2]) / (double)P->cell);
        double acc = 0.0;
        for (int i = I - ring; i <= I + ring; ++i) {
            if (i < 0 || i >= P->dims[0]) continue;
            for (int j = J - ring; j <= J + ring; ++j) {
                if (j < 0 || j >= P->dims[1]) continue;
                for (int k = K - ring; k <= K + ring; ++k) {
                    if (k < 0 || k >= P->dims[2]) continue;
                    const uint32_t c = (uint32_t)i + (uint32_t)j * P->dims[0] + (uint32_t)k * P->dims[0] * P->dims[1];
                    for (int32_t t = start[c]; t < start[c + 1]; ++t) {
                        const int32_t q = perm[t];
                        const double dx = px - pos[3 * q], dy = py - pos[3 * q + 1], dz = pz - pos[3 * q + 2];
                        const double d2 = dx * dx + dy * dy + dz * dz;
                        if (ref) {
                            const double d = sqrt(d2);
                            if (!(d <= r)) continue;
                            const float term = (1.0f / powf((float)r, 6.0f)) * powf((float)(r * r - d * d), 3.0f);
                            acc += (double)term;
                        } else {
                            const double qq = d2 / (h * h);
                            if (qq >= 1.0) continue;
                            const double w = 1.0 - qq;
                            acc += kc * (w * w * w) / rho[q];
                        }
                    }
                }
            }
        }
        iso[node] = acc;
    }
    free(keys); free(perm); free(start);
}

/* Corners (x, y, z offsets) and edges in the numbering of
 * polygonize_MarchingCube_Kernel (MarchingCube_Kernel.cu:44-56, 100-124). */
static const int MC_CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};
static const int MC_EDGE[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
static const int MC_FACE[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 3, 7, 4}, {1, 2, 6, 5}, {0, 1, 5, 4}, {3, 2, 6, 7}};

static int mc_edge_of(int a, int b) {
    for (int e = 0; e < 12; ++e)
        if ((MC_EDGE[e][0] == a && MC_EDGE[e][1] == b) || (MC_EDGE[e][0] == b && MC_EDGE[e][1] == a)) return e;
    return -1;
}

/* The case table, generated: for case bits cs (corner c set when its value is
 * <= level), each cube face joins its active edges into segments -- two
 * active edges into one segment, four (two diagonal set corners) into two
 * segments that each cut one set corner off -- and the segments close into
 * loops over the cube surface. Each loop is oriented by comparing the Newell
 * normal of its edge midpoints with the sum of (set - unset) corner offsets
 * across its edges, so triangle normals point toward the set corners, and
 * fanned from its first vertex. */
void orc_mc_table(uint8_t* ntri, int8_t* tri) {
    for (int cs = 0; cs < 256; ++cs) {
        int link[12][2], deg[12] = {0}, used[12] = {0};
        int8_t* out = &tri[cs * 30];
        for (int k = 0; k < 30; ++k) out[k] = -1;
        for (int f = 0; f < 6; ++f) {
            const int* q = MC_FACE[f];
            int act[4], na = 0;
            for (int k = 0; k < 4; ++k) {
                const int a = q[k], b = q[(k + 1) & 3];
                if (((cs >> a) & 1) != ((cs >> b) & 1)) act[na++] = mc_edge_of(a, b);
            }
            if (na == 2) {
                link[act[0]][deg[act[0]]++] = act[1];
                link[act[1]][deg[act[1]]++] = act[0];
            } else if (na == 4) {
                for (int k = 0; k < 4; ++k) {
                    if (!((cs >> q[k]) & 1)) continue;
                    const int e0 = mc_edge_of(q[(k + 3) & 3], q[k]), e1 = mc_edge_of(q[k], q[(k + 1) & 3]);
                    link[e0][deg[e0]++] = e1;
                    link[e1][deg[e1]++] = e0;
                }
            }
        }
        int nt = 0;
        for (int s0 = 0; s0 < 12; ++s0) {
            if (deg[s0] != 2 || used[s0]) continue;
            int loop[12], nl = 0, prev = -1, cur = s0;
            do {
                loop[nl++] = cur;
                used[cur] = 1;
                const int nxt = link[cur][0] != prev ? link[cur][0] : link[cur][1];
                prev = cur;
                cur = nxt;
            } while (cur != s0 && nl < 12);
            double mid[12][3], nrm[3] = {0, 0, 0}, dir[3] = {0, 0, 0};
            for (int k = 0; k < nl; ++k) {
                const int a = MC_EDGE[loop[k]][0], b = MC_EDGE[loop[k]][1];
                const int sa = (cs >> a) & 1;
                for (int d = 0; d < 3; ++d) {
                    mid[k][d] = 0.5 * (MC_CORNER[a][d] + MC_CORNER[b][d]);
                    dir[d] += sa ? MC_CORNER[a][d] - MC_CORNER[b][d] : MC_CORNER[b][d] - MC_CORNER[a][d];
                }
            }
            for (int k = 0; k < nl; ++k) {
                const double* p = mid[k];
                const double* q = mid[(k + 1) % nl];
                nrm[0] += (p[1] - q[1]) * (p[2] + q[2]);
                nrm[1] += (p[2] - q[2]) * (p[0] + q[0]);
                nrm[2] += (p[0] - q[0]) * (p[1] + q[1]);
            }
            const int flip = nrm[0] * dir[0] + nrm[1] * dir[1] + nrm[2] * dir[2] < 0;
            for (int k = 1; k + 1 < nl; ++k) {
                out[3 * nt] = (int8_t)loop[0];
                out[3 * nt + 1] = (int8_t)(flip ? loop[k + 1] : loop[k]);
                out[3 * nt + 2] = (int8_t)(flip ? loop[k] : loop[k + 1]);
                ++nt;
            }
        }
        ntri[cs] = (uint8_t)nt;
    }
}

/* vertexInterpolate_MarchingCube (MarchingCube_Kernel.cu:143-155) */
static double mc_interp(double level, double v1, double v2, double p1, double p2) {
    if (fabs(level - v1) < 0.000001) return p1;
    if (fabs(level - v2) < 0.000001) return p2;
    if (fabs(v1 - v2) < 0.000001) return p1;
    const double mu = (level - v1) / (v2 - v1);
    return p1 + mu * (p2 - p1);
}

int orc_marching_cubes(const orc_iso_grid* g, const double* iso, double level, int64_t vcap, double* vert,
                       int64_t* nv, int64_t tcap, int32_t* tri, int64_t* nt) {
    uint8_t ntri[256];
    int8_t table[256 * 30];
    orc_mc_table(ntri, table);
    const int64_t X = g->dims[0], Y = g->dims[1], Z = g->dims[2], nn = X * Y * Z;
    int64_t* vid = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)nn);
    int64_t v = 0, t = 0;
    for (int64_t node = 0; node < nn; ++node) {
        const int64_t x = node % X, y = (node / X) % Y, z = node / (X * Y);
        const int64_t step[3] = {1, X, X * Y};
        const int64_t c3[3] = {x, y, z};
        for (int a = 0; a < 3; ++a) {
            vid[3 * node + a] = -1;
            if (c3[a] + 1 >= g->dims[a]) continue;
            const double v1 = iso[node], v2 = iso[node + step[a]];
            if ((v1 <= level) == (v2 <= level)) continue;
            if (v < vcap && vert) {
                for (int d = 0; d < 3; ++d) {
                    const double p = g->origin[d] + c3[d] * g->spacing[d];
                    vert[3 * v + d] = mc_interp(level, v1, v2, p, d == a ? p + g->spacing[d] : p);
                }
            }
            vid[3 * node + a] = v++;
        }
    }
    for (int64_t node = 0; node < nn; ++node) {
        const int64_t x = node % X, y = (node / X) % Y, z = node / (X * Y);
        if (x + 1 >= X || y + 1 >= Y || z + 1 >= Z) continue;
        int cs = 0;
        for (int c = 0; c < 8; ++c) {
            const int64_t o = node + MC_CORNER[c][0] + MC_CORNER[c][1] * X + MC_CORNER[c][2] * X * Y;
            if (iso[o] <= level) cs |= 1 << c;
        }
        for (int k = 0; k < ntri[cs]; ++k, ++t) {
            if (t >= tcap || !tri) continue;
            for (int m = 0; m < 3; ++m) {
                const int e = table[cs * 30 + 3 * k + m];
                const int a = MC_EDGE[e][0], b = MC_EDGE[e][1];
                const int lo = (MC_CORNER[a][0] + MC_CORNER[a][1] + MC_CORNER[a][2]) <=
                               (MC_CORNER[b][0] + MC_CORNER[b][1] + MC_CORNER[b][2]) ? a : b;
                const int hi = lo == a ? b : a;
                const int axis = MC_CORNER[hi][0] != MC_CORNER[lo][0] ? 0 : (MC_CORNER[hi][1] != MC_CORNER[lo][1] ? 1 : 2);
                const int64_t ln = node + MC_CORNER[lo][0] + MC_CORNER[lo][1] * X + MC_CORNER[lo][2] * X * Y;
                tri[3 * t + m] = (int32_t)vid[3 * ln + axis];
            }
        }
    }
    free(vid);
    *nv = v;
    *nt = t;
    return (v > vcap || t > tcap) ? -1 : 0;
}
