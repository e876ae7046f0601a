/*
 * psb_oracle.h -- FP64 CPU restatement of the PSB particle-simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU path is compared
 * against, and the "port" CPU baseline; the product never links it.
 *
 * Pinned: in the reference-compatible profile every function here is checked
 * against the reference's own kernels executed on the CPU (oracle/_ref), see
 * tests/test_oracle_vs_reference.py. The "config" profile follows the scene
 * text (Tait EOS, penalty walls, eta loop) and has no reference counterpart.
 */
#ifndef PSB_ORACLE_H
#define PSB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_PROFILE_REF = 0, ORC_PROFILE_CONFIG = 1 };
enum { ORC_WCSPH = 0, ORC_PCISPH = 1, ORC_DEM = 2 };

typedef struct orc_params {
    int32_t n;
    float box_min[3], box_max[3];   /* container walls */
    float grid_min[3];              /* grid corner (UniformGrid.Min is float3) */
    float cell;                     /* cell edge (UniformGrid.sizeCell is float) */
    int32_t dims[3];                /* cells per axis */
    double h, mass, rho0, k, mu, sigma, l;
    float particle_radius;          /* wall offset */
    float dt;
    float gravity[3];               /* acceleration */
    int32_t profile, method;
    int32_t min_iters, max_iters;
    double eta;
    double wall_k, wall_c;          /* penalty walls: 1/s^2, 1/s */
    int32_t float_state;            /* round stored state to float like the GPU path */
    int32_t warm_start;             /* PCISPH: 0 start from p = 0, 1 start from the given p */
    double spacing;                 /* config PCISPH prototype lattice spacing (0: (m/rho0)^(1/3)) */
    double skin;                    /* config: lists hold pairs within (1 + skin) h */
    double xsph;                    /* config PCISPH: XSPH velocity smoothing factor */
    double dem_spring, dem_damping, dem_shear, dem_attraction;   /* DEM contact law */
    /* config profile: static boundary particles (Akinci et al. 2012) and
     * their volumes psi_b (kg; orc_boundary_psi); n_bnd = 0: none */
    int32_t n_bnd;
    const double* bnd_pos;      /* n_bnd * 3 */
    const double* bnd_psi;      /* n_bnd */
    /* set by the step functions: each particle's boundary neighbours at the
     * step's start positions (n x bnd_cap); NULL: every boundary particle */
    const int32_t* bnd_counts;
    const int32_t* bnd_lists;
    int32_t bnd_cap;
    /* DEM: an external force per sphere (n * 3, N; NULL: none) */
    const double* dem_ext;
    /* collision objects applied after the box walls, in order (orc_collide) */
    int32_t n_coll;
    const struct orc_collider* coll;
    /* config PCISPH, boundary particles that move with the corrector (two-
     * way coupling solved inside the step): each one's velocity and its
     * non-fluid force (gravity and contacts) at the step's start (n_bnd x 3)
     * and 1/mass; bnd_vel == NULL: the boundary is static. Each prediction
     * also predicts the boundary, x*_b = x_b + dt (v_b + dt (F_b + f_b) / m)
     * with F_b the fluid's reaction at the current pressures (at the start
     * positions, as the pressure force); the density passes see x*_b.
     * Written by the step: bnd_pred the last predicted boundary positions,
     * bnd_force the reaction F_b they were predicted with (n_bnd x 3). */
    const double* bnd_vel;
    const double* bnd_fext;
    double bnd_inv_mass;
    double* bnd_pred;
    double* bnd_force;
} orc_params;

/* One collision object of the reference (src/Kernel/Collision/*), as its
 * kernel executes. type 1 plane, 2 sphere, 3 cylinder, 4 mesh, 5 height
 * field; v[] as psb_collider's (include/psb.h). faces: count x 12 floats
 * (A, B, C, N); terms: count x 6 doubles {kind, c0..c4}, kind 1 linear
 * c0 x + c1 z, 2 Gaussian c0 exp(-((x-c1)^2/(2 c3^2) + (z-c2)^2/(2 c4^2)))
 * with the squares in float as the reference's powf, 3 cosine
 * c0 cos(c1 (x cos c2 + z sin c2) + c3). */
typedef struct orc_collider {
    int32_t type;
    int32_t container;
    float elast;
    int32_t count;
    float v[16];
    const float* faces;
    const double* terms;
} orc_collider;

/* Applies one object to n particles: old_pos the start positions (plane
 * and mesh read them), pos and vel (n x 3) updated where the object acts.
 * dt is the system's time step. Returns the number of particles moved. */
int32_t orc_collide(const orc_collider* o, int32_t n, const double* old_pos, double* pos, double* vel, float dt);

/* The force the fluid (n particles at pos with pressures p) exerts on each
 * boundary particle: minus the sum over fluid particles i within h of
 * m_i psi_b (p_i/rho0^2) 45 (h-d)^2/(pi h^6) (x_i - x_b)/d, the reaction to
 * the mirrored-pressure force. Brute force; out: nb * 3. */
void orc_boundary_reaction(const orc_params* P, const double* pos, const double* p, int32_t nb, const double* bpos,
                           const double* psi, double* out);

/* psi_b = rho0 / sum_k W(x_b - x_k) over the boundary particles within h
 * (self included), W the poly6 kernel (Akinci et al. 2012, eq. 5). */
void orc_boundary_psi(const orc_params* P, int32_t nb, const double* bpos, double* psi);

/* Pressure force density (n x 3) at pos with the given densities and
 * pressures, over the lists (n x cap), walls and boundary particles. */
void orc_pressure_force(const orc_params* P, const double* pos, const double* rho, const double* p,
                        const int32_t* counts, const int32_t* list, int32_t cap, double* fp);

/* Config-profile PCISPH pressure factor delta = 1 / (beta (|sum gradW|^2 +
 * sum |gradW|^2)) over the neighbours of a particle in a filled cubic
 * lattice of the given spacing (Solenthaler & Pajarola 2009, sec. 4). */
double orc_pci_delta(const orc_params* P);

typedef struct orc_state {
    double* pos;      /* n*3, particle-id order */
    double* vel;      /* n*3 interpolated velocity (the reference's m_dVel[1]) */
    double* vel_ap;   /* n*3 leap-frog half-step velocity (m_dVelInterAp) */
    double* rho;      /* n: density at the end of the step */
    double* p;        /* n: pressure at the end of the step */
} orc_state;

#define ORC_MAX_ITERS 64
typedef struct orc_stats {
    int32_t iters;                  /* pressure corrections performed */
    int32_t converged;
    double err[ORC_MAX_ITERS + 1];  /* max compression error per density pass */
    int64_t nbr_total;
    int32_t nbr_max;
    int32_t clamped;                /* particles whose cell was clamped into the grid */
} orc_stats;

/* SplitMix64 (Steele, Lea, Flood 2014): counter-based, so every particle's
 * jitter depends only on (seed, id, axis). */
uint64_t orc_splitmix64(uint64_t x);

/* Lattice block, ids x-fastest, positions origin + (i+0.5)*spacing + jitter
 * with jitter uniform in [-J, J), rounded once to float. xyz stride 3. */
void orc_lattice(const int32_t nxyz[3], double spacing, const double origin[3], double jitter,
                 uint64_t seed, int32_t id0, float* pos3);

/* Linear cell index i + j*nx + k*nx*ny with i = floor((x - Min)/cell) in
 * double (UniformGridKernel.cu:46-49), clamped into the grid. */
void orc_cell_keys(int32_t n, const double* pos, const float grid_min[3], float cell, const int32_t dims[3],
                   uint32_t* keys, int32_t* nclamped);

/* Stable order by (key, id): perm[t] = id of the t-th particle. */
void orc_sort_perm(int32_t n, const uint32_t* keys, int32_t* perm);

/* Neighbour lists at pos with the reference's test sqrt(d.d) <= h
 * (UniformGridKernel.cu:58-95), self included. Each list is in sorted
 * (key, id) order. Returns the total pair count, or -1 if a list would
 * exceed cap (list may be NULL to count only). */
int64_t orc_neighbors(const orc_params* P, const double* pos, int32_t cap, int32_t* counts, int32_t* list);

/* Density at pos over the lists (poly6, self included). clamp != 0 drops
 * pairs with r >= h (config profile). */
void orc_density(const orc_params* P, const double* pos, const int32_t* counts, const int32_t* list, int32_t cap,
                 int clamp, double* rho);

/* One full step (WCSPH or PCISPH per P->method) in place. Optional outputs
 * (NULL to skip): density at the step's start positions, the non-pressure
 * force density, the neighbour counts. */
int orc_step(const orc_params* P, orc_state* S, orc_stats* st, double* rho_x, double* f_np, int32_t* nbr_counts);

/* Inputs of the learned warm start at pos (config PCISPH), 7 per particle
 * in id order: see psb_oracle.c for the definitions. */
void orc_features(const orc_params* P, const double* pos, const double* vel, const double* p_prev, double* out);

/* Initial-pressure solve (PCISPH): `iters` corrector passes at eta = 0 with
 * positions and velocities restored afterwards; only S->p changes. */
int orc_presolve(const orc_params* P, orc_state* S, int32_t iters, orc_stats* st);

/* Node grid of the iso field: dims[a] nodes at origin[a] + i spacing[a], x fastest. */
typedef struct orc_iso_grid {
    double origin[3];
    double spacing[3];
    int32_t dims[3];
    double scale;      /* reference profile: influence radius h/scale over floor(1/scale) cell rings */
} orc_iso_grid;

/* Iso field at every node. Reference profile: evaluateIso_Kernel
 * (UniformGridKernel.cu:98-138). Config profile: sum_j (m/rho_j) W_poly6. */
void orc_iso_field(const orc_params* P, const double* pos, const double* rho, const orc_iso_grid* g, double* iso);

/* The generated marching-cubes case table: ntri[256], tri[256][30] (cube
 * edge numbers, -1 padded). */
void orc_mc_table(uint8_t* ntri, int8_t* tri);

/* Marching cubes at `level` over a node field: vertices on active grid edges
 * in (node, axis) order, triangles in cube order. Returns 0, or -1 when a
 * capacity is exceeded; the counts are always set. */
int orc_marching_cubes(const orc_iso_grid* g, const double* iso, double level, int64_t vcap, double* vert,
                       int64_t* nv, int64_t tcap, int32_t* tri, int64_t* nt);

#ifdef __cplusplus
}
#endif
#endif
