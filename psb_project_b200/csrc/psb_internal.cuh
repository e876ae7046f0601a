// psb_internal.cuh -- shared device-side types of libpsb (not part of the ABI).
//
// Data layout in HBM (all arrays in cell-sorted slot order after each step's
// sort; slot s holds particle ids[s]):
//   pos   float4  x, y, z, 0           16 B
//   vel   float4  interpolated v       16 B   (the reference's m_dVel[1])
//   vap   float4  leap-frog v+         16 B   (m_dVelInterAp)
//   rp    float2  (density, pressure)   8 B   (pressure persists across steps)
//   ids   int32   particle id           4 B
// Per-step scratch: sort keys/values (2 x 2 x 4 B), cell_start/cell_end
// (dense over the grid, only occupied cells are ever written or reset),
// neighbour lists (slot-major quads, see nbr_index; c < count[s]), and the
// PCISPH predictor buffers xs[2] (float4), vs (float4), rpc (float2),
// fnp (float4 non-pressure force density), rho_x (float).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include "psb.h"

namespace psb {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kBlock = 256;

struct Grid {
    float gx, gy, gz;   // corner (float, as UniformGrid.Min)
    float cell;         // edge (float, as UniformGrid.sizeCell)
    int nx, ny, nz;
};

// One scene of a batch: its box and its own grid. Every other constant is
// shared by the batch's scenes and lives in Params.
struct SceneGeom {
    float bx0, by0, bz0, bx1, by1, bz1;              // faces (ghost walls, wall distance)
    float wlo_x, wlo_y, wlo_z, whi_x, whi_y, whi_z;  // projection bounds (faces -/+ particle radius)
    Grid g;                                          // the scene's grid; its cells are keys cell_base + i + j nx + k nx ny
    uint32_t cell_base;
    int first, count;                                // its particles: sorted slots [first, first + count)
};

// Launch configuration of the tunable kernels, the autotuner's choice for a
// size bucket: block sizes (128, 256 or 512; 0 = 256) and the neighbour
// build's schedule (0: each thread walks its own 27 cells; 1: the lanes of a
// warp that share a grid row walk it together, staging candidates in shared
// memory). Every choice computes the same result bit for bit.
struct Tune {
    int nbr_block, nbr_schedule, density_block, init_block, pci_density_block, force_block, xsph_block;
};

// Uniform per-scene constants, FP32 in normalised form (q = r^2/h^2, u = r/h)
// so that no intermediate leaves FP32 range; derived on the host in FP64.
struct Collider;     // colliders.cuh

struct Params {
    int n;
    int cap;            // neighbour slots per particle
    Grid g;
    double h;           // list cut-off of the exact neighbour test sqrt(d.d) <= h in FP64
                        // (reference: h; config: (1 + skin) h)
    double h2_exact;    // the largest double x with sqrt_rn(x) <= h: the same test as d.d <= h2_exact
    float h2_lo, h2_hi; // FP32 d^2 outside [h2_lo, h2_hi] is decided without the FP64 test
    float h2, inv_h, inv_h2;
    float k_rho;        // 315 m / (64 pi h^3):           rho = k_rho * sum (1-q)^3
    float k_grad;       // 45 m / (pi h^4):               a_p = k_grad * sum (pV_i+pV_j)(1-u)^2 x^
    float k_visc;       // mu m 45 / (pi h^5):            f_v = k_visc * sum (v_j-v_i)(1-u)/rho_j
    float k_surf;       // 945 m / (32 pi h^5):           normals and surface term (reference profile)
    float sigma, l;
    float k_press;      // 1 / (beta G^2), beta = 2 (m dt/rho0)^2, G = 45/(pi h^4)
    float k_delta;      // config PCISPH: prototype delta = 1/(beta (|sum gradW|^2 + sum |gradW|^2)) of a filled lattice
    float rho0;
    double rho0_d;
    float eos_k;        // REF: k (p = k (rho - rho0));  CONFIG: k rho0 / 7 (Tait, gamma 7)
    float dt;
    float gx, gy, gz;   // gravity acceleration
    float wlo_x, wlo_y, wlo_z, whi_x, whi_y, whi_z;   // box min + r, box max - r (float, as collisionBox)
    float wall_k, wall_c;
    float xsph_k;       // config PCISPH XSPH: xsph * k_rho / rho0 (0: off)
    // DEM: contact law constants (REF: k_s, c, s, a; CONFIG: k_n, c_n), the
    // distance R in k (R - d) (REF: h_A + h_B as float; CONFIG: 2r), the
    // contact range (REF: 2R; CONFIG: 2r), sphere mass and its inverse
    float dem_k, dem_c, dem_s, dem_a, dem_R, dem_range, dem_mass, dem_inv_mass;
    int dem;
    // Config-profile walls (mirror ghost particles across the box faces):
    float bx0, by0, bz0, bx1, by1, bz1;   // faces
    float hf;           // h
    int ref;            // reference profile
    int pci;            // PCISPH (else WCSPH)
    int surface;        // surface tension on
    // Batched scenes (kernels instantiated with BATCH = true read these; the
    // box and grid fields above then go unused):
    const SceneGeom* scenes;          // per scene
    const uint16_t* slot_scene;       // scene of each sorted slot (scenes occupy contiguous slot ranges)
    const uint8_t* active;            // corrector: scenes still iterating
    unsigned long long* err_scene;    // corrector: per-scene max compression error of the pass (ordered)
    int nscenes;
    Tune tune;
    // Static boundary particles (config profile; Akinci et al. 2012): sorted
    // by cell, position in .xyz and psi_b / m in .w; per fluid slot its
    // boundary neighbours within the list cut-off, stored in quads like the
    // fluid list (bnd_cap slots). bnd_count == nullptr: no boundary.
    const float4* bnd;
    const int* bnd_count;
    const int* bnd_list;
    int bnd_cap;
    float bnd_lo[3], bnd_hi[3];     // their bounding box grown by the list cut-off
    // Boundary particles that move with the corrector (two-way coupling
    // solved inside the step): their predicted positions (psi_b / m in .w),
    // which the corrector's density passes read in place of bnd; nullptr:
    // the boundary is static.
    const float4* bnd_pred;
    // DEM: an external force per sphere in particle-id order (N; nullptr:
    // none), found through the id of each sorted slot
    const float4* ext_force;
    const int* slot_ids;
    float mass;         // particle mass (FP32)
    // Collision objects applied after the integrator and the box, in order
    // (colliders.cuh); n_coll == 0: none. Single-scene contexts only.
    const Collider* coll;
    int n_coll;
};

// Runs f(std::integral_constant<int, B>) with B the tuned block size.
template <class F>
inline void with_block(int bs, F&& f) {
    if (bs == 128) f(std::integral_constant<int, 128>{});
    else if (bs == 512) f(std::integral_constant<int, 512>{});
    else f(std::integral_constant<int, 256>{});
}

// Neighbour lists are stored in quads: entries 4q .. 4q+3 of sorted slot s
// are the int4 at index q * n + s, so one 16-byte load gives a thread four
// neighbours and a warp's 32 slots read 512 contiguous bytes per quad.
__host__ __device__ inline size_t nbr_index(int c, int n, int t) { return ((size_t)(c >> 2) * n + t) * 4 + (c & 3); }
inline size_t nbr_list_ints(size_t n, int cap) { return n * (size_t)((cap + 3) & ~3); }

// f(j) for the first cnt entries of slot t's list, in order; quads in
// flight per thread: PSB_NBR_UNROLL (a build setting). 1 measured fastest
// on B200 at 1M particles (density pass 119 us against 140 us at 2 and
// 170 us at 4): the four gathers of one quad already overlap, and fewer
// registers keep more warps resident.
#ifndef PSB_NBR_UNROLL
#define PSB_NBR_UNROLL 1
#endif
constexpr int kNbrUnroll = PSB_NBR_UNROLL;
template <class F>
__device__ __forceinline__ void for_each_nbr(const int* __restrict__ list, int n, int t, int cnt, F&& f) {
    const int4* __restrict__ L = reinterpret_cast<const int4*>(list) + t;
    int c = 0;
#pragma unroll kNbrUnroll
    for (; c + 4 <= cnt; c += 4) {
        const int4 q = __ldg(L + (size_t)(c >> 2) * n);
        f(q.x); f(q.y); f(q.z); f(q.w);
    }
    if (c < cnt) {
        const int4 q = __ldg(L + (size_t)(c >> 2) * n);
        f(q.x);
        if (c + 1 < cnt) f(q.y);
        if (c + 2 < cnt) f(q.z);
    }
}

// |d|^2 of a pair in FP32 with the multiply-adds written out, so that every
// kernel that tests or weights the same pair rounds it the same way.
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// The reference's test, sqrt((dx*dx + dy*dy) + dz*dz) <= h with every
// operation rounded separately in FP64 (double3.h:15-47). The correctly
// rounded square root is monotone, so the test is d2 <= h2_exact, the
// largest double whose root rounds to at most h (found on the host).
__device__ __forceinline__ bool exact_neighbor(float4 a, float4 b, double h2_exact) {
    const double dx = __dsub_rn((double)a.x, (double)b.x);
    const double dy = __dsub_rn((double)a.y, (double)b.y);
    const double dz = __dsub_rn((double)a.z, (double)b.z);
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return d2 <= h2_exact;
}

// flags[1]: max count, flags[2..3]: total pairs (64-bit); every lane of the
// warp calls it.
__device__ __forceinline__ void nbr_flags(int cnt, int* __restrict__ flags) {
    int m = cnt;
    unsigned long long tot = (unsigned long long)cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if ((threadIdx.x & 31) == 0 && tot > 0) {
        atomicMax(&flags[1], m);
        atomicAdd((unsigned long long*)&flags[2], tot);
    }
}

// The 27-cell walk of sorted particle t (one thread per particle): the three
// cells of a grid row are adjacent in sorted order, so each of the nine rows
// is one contiguous slot range, and accept(slot, position) runs for every
// candidate within the list cut-off in increasing slot order, row by row --
// the list order. In a batch the walk stays inside the particle's scene's
// grid. Candidates beyond the FP32 window are out with one compare, those
// below it in; inside it the reference's FP64 test decides.
template <bool BATCH, class F>
__device__ __forceinline__ void walk_neighbours(const Params& P, int t, float4 pi, const float4* __restrict__ pos,
                                                const uint32_t* __restrict__ keys,
                                                const uint32_t* __restrict__ cell_start,
                                                const uint32_t* __restrict__ cell_end, F&& accept) {
    const Grid g = BATCH ? P.scenes[P.slot_scene[t]].g : P.g;
    const uint32_t base = BATCH ? P.scenes[P.slot_scene[t]].cell_base : 0u;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const uint32_t key = keys[t] - base;
    const int ci = (int)(key % (uint32_t)nx);
    const int cj = (int)((key / (uint32_t)nx) % (uint32_t)ny);
    const int ck = (int)(key / ((uint32_t)nx * (uint32_t)ny));
    // Skipping the cells whose faces lie beyond the cut-off (a bound from the
    // particle's distance to its own cell's faces) was measured: the lanes of
    // a warp prune different cells, so the warp still walks their union, and
    // the per-row bounds cost more than the skipped candidates save.
    const int a0 = max(ci - 1, 0), a1 = min(ci + 1, nx - 1);
    for (int k = max(ck - 1, 0); k <= min(ck + 1, nz - 1); ++k) {
        for (int j = max(cj - 1, 0); j <= min(cj + 1, ny - 1); ++j) {
            const uint32_t row = base + (uint32_t)j * (uint32_t)nx + (uint32_t)k * (uint32_t)nx * (uint32_t)ny;
            uint32_t lo = kEmpty, hi = 0;
            for (int a = a0; a <= a1; ++a) {
                const uint32_t s = cell_start[row + a];
                if (s != kEmpty) {
                    if (lo == kEmpty) lo = s;
                    hi = cell_end[row + a];
                }
            }
            if (lo == kEmpty) continue;
            for (uint32_t q = lo; q < hi; ++q) {
                const float4 pj = pos[q];
                const float d2 = dist2(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z);
                if (d2 <= P.h2_hi && (d2 < P.h2_lo || exact_neighbor(pi, pj, P.h2_exact))) accept(q, pj);
            }
        }
    }
}

// ---- launchers (grid.cu) -------------------------------------------------
void launch_reset_cells(cudaStream_t st, int n, const uint32_t* sorted_keys, uint32_t* cell_start);
void launch_cell_keys(cudaStream_t st, const Params& P, const float4* pos, const int* ids, uint32_t* keys_by_id,
                      uint32_t* slot_by_id, int* clamped);
// Sorts (keys, vals) by key, stably; returns the buffer index (0 or 1) holding the result.
// hist holds 256 * radix_blocks(n) + 256 words.
int radix_sort(cudaStream_t st, int n, int bits, uint32_t* keys[2], uint32_t* vals[2], uint32_t* hist, int nblocks_cap);
int radix_blocks(int n);
// The whole state into sorted order, with the cell ranges; or in two
// launches: positions, ids and cell ranges (what the neighbour build reads),
// then the rest.
void launch_reorder(cudaStream_t st, int n, const uint32_t* keys, const uint32_t* vals, const float4* pos,
                    const float4* vel, const float4* vap, const float2* rp, const int* ids, float4* pos2, float4* vel2,
                    float4* vap2, float2* rp2, int* ids2, uint32_t* cell_start, uint32_t* cell_end);
void launch_reorder_pos(cudaStream_t st, int n, const uint32_t* keys, const uint32_t* vals, const float4* pos,
                        const int* ids, float4* pos2, int* ids2, uint32_t* cell_start, uint32_t* cell_end);
void launch_reorder_state(cudaStream_t st, int n, const uint32_t* vals, const float4* vel, const float4* vap,
                          const float2* rp, float4* vel2, float4* vap2, float2* rp2);
void launch_build_nbr(cudaStream_t st, const Params& P, const float4* pos, const uint32_t* keys,
                      const uint32_t* cell_start, const uint32_t* cell_end, int* counts, int* list, int* flags);
// (sph.cu) The per-thread neighbour build of one config-profile scene with the
// density pass at x folded in: lists, counts and flags as launch_build_nbr,
// then density, pressure and features as launch_density_x.
void launch_build_density(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const uint32_t* keys,
                          const uint32_t* cell_start, const uint32_t* cell_end, int* counts, int* list, int* flags,
                          float2* rp, float* rho_x, int zero_p, float p_scale, float* feats, int nfeat);

// ---- launchers (sph.cu) ---------------------------------------------------
// feats != nullptr: also the warm start's inputs f0 .. f(nfeat - 1), nfeat 6 or 7.
void launch_density_x(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                      const int* list, float2* rp, float* rho_x, int zero_p, float p_scale = 1.f,
                      float* feats = nullptr, int nfeat = 7);
void launch_wcsph_force(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const float4* vap,
                        const float2* rp, const int* counts, const int* list, float4* pos_out, float4* vel_out,
                        float4* vap_out, float4* fnp);
void launch_pci_init(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const float4* vap,
                     const float2* rp, const int* counts, const int* list, int warm, float4* fnp, float4* xs,
                     float4* vs);
void launch_pci_density(cudaStream_t st, const Params& P, const float4* xs, const float2* rp, const int* counts,
                        const int* list, float2* rpc, unsigned long long* err_slot);
void launch_pci_force_predict(cudaStream_t st, const Params& P, const float4* pos, const float4* vap,
                              const float4* fnp, const float4* xs, const float2* rpc, const int* counts,
                              const int* list, float4* xs_next, float4* vs, float2* rp);
void launch_pci_commit(cudaStream_t st, const Params& P, const float4* xs, const float4* vs, const float2* rpc,
                       int have_density_pass, float4* pos, float4* vel, float4* vap, float2* rp);
void launch_xsph(cudaStream_t st, const Params& P, const float4* xs, const float4* vs, const int* counts,
                 const int* list, float4* vs_out);
void launch_dem_step(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                     const int* list, float4* pos_out, float4* vel_out, float4* vap_out, float4* force);
// The force on each sphere (slot order) that the next step would apply
// without its external force: gravity and the contacts; nothing moves.
void launch_dem_forces(cudaStream_t st, const Params& P, const float4* pos, const float4* vel, const int* counts,
                       const int* list, float4* force);

// ---- batched scenes: the corrector loop on the device (batch.cu) ---------------
// loop: [0] pass index, [1] continue, [2, 2 + S) corrections, [2 + S, 2 + 2S) converged,
// [2 + 2S, 2 + 3S) corrections summed over steps, [2 + 3S, 2 + 4S) unconverged steps
void launch_batch_begin(cudaStream_t st, int S, int max_it, uint8_t* active, unsigned long long* err_scene,
                        unsigned long long* err_hist, int hist_len, int* loop);
void launch_batch_decide(cudaStream_t st, int S, int min_it, int max_it, double eta, uint8_t* active,
                         unsigned long long* err_scene, unsigned long long* err_hist, int* loop,
                         cudaGraphConditionalHandle handle, int set_handle);
// The whole corrector loop of a config-profile scene or batch as one
// cooperative launch (begin, then {density pass, decision, pressure-force
// pass} until the decision ends it). Returns the launch's error.
cudaError_t launch_corrector_persistent(cudaStream_t st, const Params& P, const float4* pos, const float4* vap,
                                        const float4* fnp, float4* xs, float2* rp, float2* rpc, const int* counts,
                                        const int* list, float4* vs, int S, int min_it, int max_it, double eta,
                                        uint8_t* active, unsigned long long* err_scene, unsigned long long* err_hist,
                                        int* loop);

// ---- boundary particles (boundary.cu) ------------------------------------------
// Sorts nb boundary particles by cell (stable on index), fills their cell
// ranges and writes psi_b / m to .w of sorted[]: rho0 / (k_rho sum_k (1 -
// q_bk)^3) over the boundary particles within h, self included. Returns the
// buffer (0 or 1) of keys[] that holds the sorted keys.
int launch_bnd_prepare(cudaStream_t st, const Params& P, int nb, const float4* raw, int* iota, uint32_t* keys[2],
                       uint32_t* vals[2], uint32_t* hist, int hist_blocks, int key_bits, float4* sorted, int* ids,
                       float* w, uint32_t* cell_start, uint32_t* cell_end, int* clamped);
// The force the fluid exerts on each sorted boundary particle: minus the sum
// of the mirrored-pressure forces the particle exerts on the fluid within h,
// from the fluid's positions and committed pressures (sorted slots, cell
// ranges of the last build). Written as float4 per boundary slot.
// Collision objects on the integrator's output (WCSPH and DEM; the PCISPH
// commit applies them itself). x_old: the step's start positions. vh_old
// (WCSPH): the start half-step velocities, for v = (vh_old + vap)/2; null
// (DEM): vel and vap both take the new velocity.
void launch_apply_colliders(cudaStream_t st, const Params& P, const float4* x_old, const float4* vh_old, float4* pos,
                            float4* vel, float4* vap);
// Emission (emit.cu): k particles at slots and ids n0 .. n0 + k - 1, velocity
// v, half-step velocity v (dem) or 0, density and pressure 0.
void launch_emit_list(cudaStream_t st, int n0, int k, const float* xyz, const float* v, int dem, float4* pos,
                      float4* vel, float4* vap, int* ids, float2* rp);
void launch_emit_random(cudaStream_t st, int n0, int k, int type, int count, unsigned emission,
                        unsigned long long seed, const float* params, const float* faces, const float* v, int dem,
                        float4* pos, float4* vel, float4* vap, int* ids, float2* rp);
void launch_append_ids(cudaStream_t st, int n0, int k, int* ids, float2* rp);
void launch_bnd_reaction(cudaStream_t st, const Params& P, int nb, const float4* fluid_pos, const float2* fluid_rp,
                         const uint32_t* cell_start, const uint32_t* cell_end, float4* force);
// Moving boundary (sorted slots): the reaction F_b at the pressures in
// fluid_rp (fluid at the step's start positions) into force, and the
// prediction x*_b = x_b + dt (v_b + dt (F_b + f_b) / m) into pred (.w:
// psi_b / m, from P.bnd).
void launch_bnd_move(cudaStream_t st, const Params& P, int nb, const float4* fluid_pos, const float2* fluid_rp,
                     const uint32_t* cell_start, const uint32_t* cell_end, const float4* vel, const float4* fext,
                     float inv_mass, float4* pred, float4* force);
// dst[t] = src[ids[t]] (boundary arrays from their input order to sorted slots)
void launch_bnd_gather4(cudaStream_t st, int nb, const int* ids, const float4* src, float4* dst);
// Per fluid slot: the boundary particles within the list cut-off, from a
// 27-cell walk of the boundary's cell ranges (none outside P.bnd_lo/hi);
// flags[0] is set when a slot has more than P.bnd_cap.
void launch_build_bnd_nbr(cudaStream_t st, const Params& P, const float4* pos, const uint32_t* keys,
                          const uint32_t* bnd_start, const uint32_t* bnd_end, int* counts, int* list, int* flags);

// ---- FP64 diagnostics (diag.cu) -------------------------------------------------
// terms: mass, momentum x/y/z, kinetic, potential, sum and max of |rho - rho0|/rho0
constexpr int kDiagTerms = 8;
int diag_rows(int count);
void launch_diagnostics(cudaStream_t st, int first, int count, double mass, double rho0, const float g[3],
                        const float4* pos, const float4* vel, const float2* rp, double* rows, double* out);

// ---- iso field and marching cubes (mc.cu) ----------------------------------------
constexpr int kMcMaxTri = 10;       // at most 12 active edges in loops of >= 3: 12 - 2 triangles
struct IsoParams {
    double origin[3];   // node (0, 0, 0)
    double spacing[3];  // node spacing per axis
    int dims[3];        // nodes per axis
    double level;       // iso level of the surface
    double r;           // REF: influence radius h / scale
    int ring;           // cells of the particle grid walked on each side of the node's cell
    double inv_r2;      // CONFIG: 1 / h^2
    double k_colour;    // CONFIG: m 315 / (64 pi h^3): c(x) = k_colour sum (1 - q)^3 / rho_j
};
void mc_build_table(uint8_t ntri[256], int8_t tri[256][kMcMaxTri * 3]);
void mc_upload_table(cudaStream_t st);
long long scan_scratch_words(long long n);
void scan_exclusive_u32(cudaStream_t st, long long n, uint32_t* data, uint32_t* scratch);
void launch_iso_field(cudaStream_t st, const IsoParams& Q, const Params& P, const float4* pos, const float2* rp,
                      const uint32_t* cell_start, const uint32_t* cell_end, double* iso);
void launch_mc_classify(cudaStream_t st, const IsoParams& Q, const double* iso, uint32_t* cube_tris,
                        uint32_t* edge_flag);
void launch_mc_emit(cudaStream_t st, const IsoParams& Q, const double* iso, const uint32_t* edge_off,
                    const uint32_t* tri_off, float* vert, int32_t* tris);
// The reference's polygonizer layout (compat): double4 nodes, per-cube vertex
// slots and counts; synchronous, reports a slot overflow on stderr.
void launch_mc_polygonize_slots(cudaStream_t st, const double* node4, int nx, int ny, int nz, double level, int* count,
                                double* vertex, int* index, int slots);

// ---- learned warm start (mlp.cu) ---------------------------------------------------
// Networks (psb.h PSB_MLP_*): arch 0 6 -> 64 -> 64 -> 1 SiLU, arch 1 7 -> 64 -> 64 -> 1 ReLU.
constexpr int kMlpParams = 4737;   // the larger network's parameters: 7x64 + 64 + 64x64 + 64 + 64 + 1
int mlp_inputs(int arch);
int mlp_params(int arch);
void launch_mlp_infer(cudaStream_t st, int arch, int n, const float* feats, const void* wbf, float p_scale, float2* rp);
void launch_mlp_forward(cudaStream_t st, int arch, int n, const float* X, const void* wbf, float* y);
// Training blocks per minibatch (at most) and the gradient partials they
// write: kMlpGradBlocks rows of kMlpParams + 1 floats (the caller's buffer).
constexpr int kMlpGradBlocks = 148 * 4;
constexpr size_t kMlpGradPartials = (size_t)kMlpGradBlocks * (kMlpParams + 1);
void launch_mlp_grad(cudaStream_t st, int arch, int batch, const float* X, const float* T, const uint32_t* sel,
                     const void* wbf, float* partial, float* grad, float* loss);
void launch_mlp_sample(cudaStream_t st, int batch, uint64_t size, uint64_t seed, uint32_t* sel);
void launch_adam(cudaStream_t st, int np, float* w, const float* grad, float* m1, float* m2, void* wbf, float lr,
                 int step);
void launch_to_bf16(cudaStream_t st, int np, const float* w, void* wbf);
void launch_collect(cudaStream_t st, int n, int stride, int offset, uint64_t base, uint64_t cap, const float* feats,
                    const float2* rp, float p_scale, float* X, float* T);
void launch_zero_pressure(cudaStream_t st, int n, float2* rp);

// Ordered encoding of doubles for atomicMax on unsigned 64-bit words.
__host__ __device__ inline unsigned long long order_double(double v) {
    long long b;
#ifdef __CUDA_ARCH__
    b = __double_as_longlong(v);
#else
    __builtin_memcpy(&b, &v, 8);
#endif
    return b >= 0 ? (unsigned long long)b ^ 0x8000000000000000ull : ~(unsigned long long)b;
}
__host__ __device__ inline double unorder_double(unsigned long long u) {
    long long b = (u & 0x8000000000000000ull) ? (long long)(u ^ 0x8000000000000000ull) : (long long)~u;
    double v;
#ifdef __CUDA_ARCH__
    v = __longlong_as_double(b);
#else
    __builtin_memcpy(&v, &b, 8);
#endif
    return v;
}

// Start of a step's corrector, run by one block. With max_iters = 0 no pass
// runs and every scene ends unconverged with no corrections, as a single
// scene does.
__device__ inline void corrector_begin(int S, int max_it, uint8_t* active, unsigned long long* err_scene,
                                       unsigned long long* err_hist, int hist_len, int* loop) {
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        active[s] = 1;
        err_scene[s] = 0ull;
        loop[2 + s] = 0;
        loop[2 + S + s] = 0;
        if (max_it == 0) loop[2 + 3 * S + s] += 1;
    }
    for (int i = threadIdx.x; i < hist_len; i += blockDim.x) err_hist[i] = 0ull;
    if (threadIdx.x == 0) { loop[0] = 0; loop[1] = 1; }
}

// After density pass k, run by one block (every thread calls it; any is a
// shared word). A scene converges when k >= min_iters and its error is at
// most eta (the host loop's test, in FP64 on the same value). A scene that
// has not converged takes the pressure-force pass; if that pass is its
// max_iters-th, it stops after it, unconverged, with max_iters corrections.
// Returns (to every thread) whether another pass follows.
__device__ inline int corrector_decide(int S, int min_it, int max_it, double eta, uint8_t* active,
                                       unsigned long long* err_scene, unsigned long long* err_hist, int* loop,
                                       int* any) {
    if (threadIdx.x == 0) *any = 0;
    __syncthreads();
    const int k = loop[0];
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        if (!active[s]) continue;
        const unsigned long long e = err_scene[s];
        if (k < PSB_MAX_ITERS + 1) err_hist[(size_t)k * S + s] = e;
        err_scene[s] = 0ull;
        if (k >= min_it && e != 0ull && unorder_double(e) <= eta) {
            active[s] = 0;
            loop[2 + s] = k;
            loop[2 + S + s] = 1;
            loop[2 + 2 * S + s] += k;
        } else if (k + 1 >= max_it) {
            loop[2 + s] = k + 1;          // last pass; stays active for it
            loop[2 + 2 * S + s] += k + 1;
            loop[2 + 3 * S + s] += 1;
        } else {
            *any = 1;
        }
    }
    __syncthreads();
    // k + 1 < max_it <= PSB_MAX_ITERS whenever any is set: the loop ends
    const int cont = *any && k + 1 < max_it && k + 1 <= PSB_MAX_ITERS;
    __syncthreads();
    if (threadIdx.x == 0) {
        loop[0] = k + 1;
        loop[1] = cont;
    }
    return cont;
}


}  // namespace psb
