// api.cu -- the C ABI (include/psb.h): context, buffers, step orchestration,
// uploads/downloads in particle-id order, per-kernel CUDA-event profiling.
//
// One psb_step is, on the context's stream:
//   reset cells of the previous sort -> cell keys -> radix sort (cell, id) ->
//   reorder + cell ranges -> neighbour lists -> density at x ->
//   WCSPH: forces + leap-frog + walls + interpolation (one sweep)
//   PCISPH: non-pressure forces + first prediction, then per correction
//           {density/pressure pass at x*, pressure-force pass + next
//           prediction}, then commit + walls + interpolation.
// The reference profile runs exactly three corrections with no host
// round-trip; the config profile reads the FP64 max compression error of
// each density pass (8 bytes) to decide convergence.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <map>

#include "psb.h"
#include "psb_internal.cuh"
#include "colliders.cuh"
#include "emitters.h"

using psb::Params;

namespace {

struct Profiler {
    bool on = false;
    std::vector<std::string> names;
    std::vector<long long> launches;
    std::vector<double> ms;
    struct Pending { int k; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;

    int index(const char* name) {
        for (size_t i = 0; i < names.size(); ++i)
            if (names[i] == name) return (int)i;
        names.emplace_back(name);
        launches.push_back(0);
        ms.push_back(0.0);
        return (int)names.size() - 1;
    }
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void resolve(cudaStream_t st) {
        if (pending.empty()) return;
        cudaStreamSynchronize(st);
        for (auto& p : pending) {
            float t = 0.f;
            cudaEventElapsedTime(&t, p.a, p.b);
            launches[p.k] += 1;
            ms[p.k] += t;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    ~Profiler() {
        for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

}  // namespace

// One emitter (psb_add_emitter): the deterministic types keep their
// emission's positions on the device; the random ones keep mesh faces.
struct EmitterRec {
    psb_emitter e{};
    float* d_list = nullptr;
    float* d_faces = nullptr;
    int64_t per = 0;      // particles per emission
    int done = 0;         // emissions so far
};

struct psb_ctx {
    psb_scene sc{};
    Params P{};
    int device = 0;
    int n = 0, n_max = 0, cap = 0;
    cudaStream_t stream = nullptr;
    // particle state, double-buffered for the reorder: cs indexes pos/vel/vap,
    // cr indexes rp/ids
    float4* pos[2] = {};
    float4* vel[2] = {};
    float4* vap[2] = {};
    float2* rp[2] = {};
    int* ids[2] = {};
    int cs = 0, cr = 0;
    // sort and cells
    uint32_t* keys[2] = {};
    uint32_t* vals[2] = {};
    uint32_t* hist = nullptr;
    int hist_blocks = 0, key_bits = 0;
    int sorted = -1;          // buffer holding the last sorted keys, -1: none
    int sorted_n = 0;
    int stale = -1;           // after an upload: the previous particle set's sorted keys, whose cells
    int stale_n = 0;          // the next build clears (-1: none)
    uint32_t* cell_start = nullptr;
    uint32_t* cell_end = nullptr;
    size_t ncells = 0;
    int* nbr_count = nullptr;
    int* nbr_list = nullptr;
    // SPH scratch
    float4* fnp = nullptr;
    float4* xs[2] = {};
    float4* vs = nullptr;
    float2* rpc = nullptr;
    float* rho_x = nullptr;
    unsigned long long* err_hist = nullptr;
    int* flags = nullptr;     // [0] overflow [1] max count [2..3] pair total [4] clamped
    void* stage = nullptr;    // device staging for uploads/downloads
    // learned warm start
    float* feats = nullptr;   // n_max x 8
    float* mlp_w = nullptr;   // FP32 master weights
    float* mlp_m1 = nullptr;
    float* mlp_m2 = nullptr;
    float* mlp_grad = nullptr;
    float* mlp_part = nullptr;    // per-block gradient partials (summed in block order)
    float* mlp_loss = nullptr;
    void* mlp_wbf = nullptr;  // BF16 copy used by the kernels
    int mlp_step = 0;
    bool mlp_set = false;
    int mlp_arch = PSB_MLP_SILU6;   // the network (psb_mlp_set_arch)
    float p_scale = 1.f;
    float* ds_X = nullptr;    // recorded rows x 8
    float* ds_T = nullptr;
    uint64_t ds_cap = 0, ds_rows = 0;
    int collect_stride = 0;
    int64_t collect_steps = 0;
    uint32_t* sel = nullptr;
    int sel_cap = 0;
    // iso field and marching cubes (grown on demand)
    double* iso = nullptr;
    uint32_t* mc_cube = nullptr;   // per-node triangle counts -> offsets
    uint32_t* mc_edge = nullptr;   // per-edge flags -> vertex offsets
    uint32_t* mc_scratch = nullptr;
    float* mc_vert = nullptr;
    int32_t* mc_tri = nullptr;
    long long iso_cap = 0, mc_cube_cap = 0, mc_edge_cap = 0, mc_scratch_cap = 0, mc_vert_cap = 0, mc_tri_cap = 0;
    bool mc_table = false;
    // batched scenes (psb_create_batch); a single scene has nscenes == 1 and batch == false
    bool batch = false;
    int nscenes = 1;
    std::vector<int64_t> first{0, 0};        // first particle id of each scene, then the total
    std::vector<psb::SceneGeom> geom;
    psb::SceneGeom* d_scenes = nullptr;
    uint16_t* d_slot_scene = nullptr;
    uint8_t* d_active = nullptr;
    unsigned long long* d_err_scene = nullptr;    // the current density pass, per scene
    unsigned long long* d_err_sh = nullptr;       // (PSB_MAX_ITERS + 1) x nscenes, per pass and scene
    int* d_loop = nullptr;                        // device loop words (batch.cu)
    int* h_loop = nullptr;                        // pinned mirrors
    unsigned long long* h_err_sh = nullptr;
    // DEM: external force per sphere (psb_set_external_force), id order
    float4* ext_force = nullptr;
    float4* bnd_force = nullptr;    // boundary reaction scratch (psb_boundary_forces)
    // collision objects (psb_set_colliders): the device list and each
    // object's mesh faces or height terms
    psb::Collider* d_coll = nullptr;
    std::vector<float*> coll_data;
    std::vector<EmitterRec> emitters;     // psb_add_emitter, in order
    long long bnd_force_cap = 0;
    // static boundary particles (psb_set_boundary); bnd_n == 0: none
    int bnd_n = 0, bnd_res = 0;
    static constexpr int kBndCap = 64;
    float4* bnd_raw = nullptr;
    float4* bnd_sorted = nullptr;
    int* bnd_ids = nullptr;
    int* bnd_iota = nullptr;
    float* bnd_w = nullptr;
    uint32_t* bnd_keys[2] = {};
    uint32_t* bnd_vals[2] = {};
    uint32_t* bnd_hist = nullptr;
    uint32_t* bnd_cs = nullptr;     // boundary cell ranges over the grid
    uint32_t* bnd_ce = nullptr;
    int* bnd_count = nullptr;       // per fluid slot
    int* bnd_list = nullptr;
    long long bnd_cap_alloc = 0;
    // boundary moving with the corrector (psb_set_boundary_motion), per
    // sorted boundary slot: velocity and non-fluid force at the step's start,
    // the predicted positions and the reaction they were predicted with
    bool bnd_moving = false;
    float bnd_inv_mass = 0.f;
    float4* bnd_vel = nullptr;
    float4* bnd_fext = nullptr;
    float4* bnd_pred = nullptr;
    float4* bnd_react = nullptr;
    long long bnd_motion_cap = 0;
    // the context's own stream-ordered pool for the buffers that grow on
    // demand (grow); it keeps freed memory for the next growth
    cudaMemPool_t pool = nullptr;
    // FP64 diagnostics scratch (grown on demand)
    double* diag_rows = nullptr;
    double* diag_out = nullptr;
    long long diag_rows_cap = 0, diag_out_cap = 0;
    // autotuner: launch configuration per size bucket (floor(log2 n))
    std::map<int, psb_tune> tune_table;
    // CUDA-graph stepping (batches)
    bool graph_on = false;
    int corrector = PSB_CORRECTOR_LAUNCHES;       // the corrector loop: kernel per pass, or one persistent launch
    // one per state buffer parity (cs), plain [0, 1] and for the first step
    // after an upload [2, 3] (its state gather waits for the upload's copies)
    cudaGraphExec_t gexec[4] = {};
    bool capture_split = false;                   // the kind of graph being captured
    int graph_sorted = -1;                        // the sort's result buffer, fixed by the key width
    int graph_n = -1;                             // the particle count the graphs were captured for
    int64_t iters_total_base = 0;                 // single scene: corrections before the loop words' sums
    cudaStream_t cap_main = nullptr;              // captures the step (the legacy stream cannot be captured)
    cudaStream_t cap_stream = nullptr;            // captures the while node's body
    // psb_upload copies velocities and pressures on copy_st while the next
    // step's grid and neighbour build run; ev_in marks them in place, and the
    // step waits for it only where it gathers them (in_pending: not yet
    // waited for on the context's stream)
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_in = nullptr;
    cudaEvent_t ev_tail = nullptr;                // orders one stream after another's queued work
    bool in_pending = false;
    // host mirrors
    unsigned long long* h_err = nullptr;
    int* h_flags = nullptr;
    bool uploaded = false, built = false;
    psb_step_stats stats{};
    Profiler prof;
    std::string err;
};

namespace {

const char* kStatus[] = {"ok", "invalid argument", "out of memory", "neighbour list overflow",
                         "corrector did not converge", "CUDA error", "call out of order"};

int fail(psb_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_check(psb_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PSB_OK;
    return fail(c, PSB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PSB_TRY(expr)                          \
    do {                                       \
        int rc__ = (expr);                     \
        if (rc__ != PSB_OK) return rc__;       \
    } while (0)

template <typename F>
void timed(psb_ctx* c, const char* name, F&& launch) {
    if (!c->prof.on) { launch(); return; }
    const int k = c->prof.index(name);
    cudaEvent_t a = c->prof.get(), b = c->prof.get();
    cudaEventRecord(a, c->stream);
    launch();
    cudaEventRecord(b, c->stream);
    c->prof.pending.push_back({k, a, b});
    if (c->prof.pending.size() > 8192) c->prof.resolve(c->stream);
}

// Stream `to` runs after the work queued on `from` so far.
int follow(psb_ctx* c, cudaStream_t from, cudaStream_t to) {
    cudaError_t e = cudaEventRecord(c->ev_tail, from);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(to, c->ev_tail, 0);
    return cuda_check(c, e, "stream order");
}

// The context's stream waits for the last upload's copies on the copy
// stream. Every entry point runs it first, except psb_step, whose step waits
// at the first kernel that reads those arrays (wait_inputs).
void join_inputs(psb_ctx* c) {
    if (!c->in_pending) return;
    cudaStreamWaitEvent(c->stream, c->ev_in, 0);
    c->in_pending = false;
}

void enter(psb_ctx* c) {
    cudaSetDevice(c->device);
    join_inputs(c);
}

bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    return cs == cudaStreamCaptureStatusActive;
}

// Inside a step, before the first kernel that reads the uploaded velocities
// or pressures. A step being captured into a graph gets an external event
// wait node: each launch of the graph then waits for the record of ev_in
// that precedes it (the last upload's).
void wait_inputs(psb_ctx* c, cudaStream_t st) {
    if (capturing(st)) {
        cudaStreamWaitEvent(st, c->ev_in, cudaEventWaitExternal);
        return;
    }
    join_inputs(c);
}

template <typename T>
int dalloc(psb_ctx* c, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc((void**)p, sizeof(T) * count) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, PSB_ENOMEM, "cudaMalloc of " + std::to_string(sizeof(T) * count) + " bytes failed");
    }
    return PSB_OK;
}

void free_all(psb_ctx* c) {
    for (int i = 0; i < 2; ++i) {
        cudaFree(c->pos[i]); cudaFree(c->vel[i]); cudaFree(c->vap[i]); cudaFree(c->rp[i]); cudaFree(c->ids[i]);
        cudaFree(c->keys[i]); cudaFree(c->vals[i]); cudaFree(c->xs[i]);
    }
    cudaFree(c->hist); cudaFree(c->cell_start); cudaFree(c->cell_end); cudaFree(c->nbr_count);
    cudaFree(c->nbr_list); cudaFree(c->fnp); cudaFree(c->vs); cudaFree(c->rpc); cudaFree(c->rho_x);
    cudaFree(c->err_hist); cudaFree(c->flags); cudaFree(c->stage);
    cudaFree(c->bnd_vel); cudaFree(c->bnd_fext); cudaFree(c->bnd_pred); cudaFree(c->bnd_react);
    cudaFree(c->feats); cudaFree(c->mlp_w); cudaFree(c->mlp_m1); cudaFree(c->mlp_m2); cudaFree(c->mlp_grad); cudaFree(c->mlp_part);
    cudaFree(c->mlp_loss); cudaFree(c->mlp_wbf); cudaFree(c->ds_X); cudaFree(c->ds_T); cudaFree(c->sel);
    cudaFree(c->iso); cudaFree(c->mc_cube); cudaFree(c->mc_edge); cudaFree(c->mc_scratch); cudaFree(c->mc_vert);
    cudaFree(c->mc_tri);
    cudaFreeHost(c->h_err); cudaFreeHost(c->h_flags);
    cudaFree(c->d_scenes); cudaFree(c->d_slot_scene); cudaFree(c->d_active); cudaFree(c->d_err_scene);
    cudaFree(c->d_err_sh); cudaFree(c->d_loop);
    cudaFree(c->diag_rows); cudaFree(c->diag_out);
    cudaFree(c->bnd_raw); cudaFree(c->bnd_sorted); cudaFree(c->bnd_ids); cudaFree(c->bnd_iota); cudaFree(c->bnd_w);
    for (int i = 0; i < 2; ++i) { cudaFree(c->bnd_keys[i]); cudaFree(c->bnd_vals[i]); }
    cudaFree(c->bnd_hist); cudaFree(c->bnd_cs); cudaFree(c->bnd_ce); cudaFree(c->bnd_count); cudaFree(c->bnd_list);
    cudaFree(c->ext_force); cudaFree(c->bnd_force);
    cudaFree(c->d_coll);
    for (float* d : c->coll_data) cudaFree(d);
    for (auto& e : c->emitters) { cudaFree(e.d_list); cudaFree(e.d_faces); }
    cudaFreeHost(c->h_loop); cudaFreeHost(c->h_err_sh);
    for (auto& g : c->gexec) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->cap_main) cudaStreamDestroy(c->cap_main);
    if (c->copy_st) cudaStreamDestroy(c->copy_st);
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    if (c->ev_tail) cudaEventDestroy(c->ev_tail);
    if (c->pool) cudaMemPoolDestroy(c->pool);
}

int validate(const psb_scene* s, std::string& why) {
    if (!s) { why = "scene is NULL"; return PSB_EINVAL; }
    if (s->n_max <= 0) { why = "n_max must be positive"; return PSB_EINVAL; }
    if (!(s->h > 0) || !(s->mass > 0) || !(s->rho0 > 0) || !(s->dt > 0)) { why = "h, mass, rho0, dt must be positive"; return PSB_EINVAL; }
    if (!(s->skin >= 0) || (s->profile == PSB_PROFILE_REF && s->skin != 0)) { why = "skin must be >= 0 (0 in the reference profile)"; return PSB_EINVAL; }
    if (!(s->xsph >= 0 && s->xsph <= 1) || (s->profile == PSB_PROFILE_REF && s->xsph != 0)) { why = "xsph must be in [0, 1] (0 in the reference profile)"; return PSB_EINVAL; }
    if (!(s->cell > 0) || (double)s->cell < s->h * (1.0 + s->skin) * (1.0 - 1e-6)) {
        why = "cell must be >= (1 + skin) h (27-cell walk)";
        return PSB_EINVAL;
    }
    for (int a = 0; a < 3; ++a) {
        if (s->dims[a] <= 0) { why = "dims must be positive"; return PSB_EINVAL; }
        if (!(s->box_max[a] > s->box_min[a])) { why = "box_max must exceed box_min"; return PSB_EINVAL; }
    }
    const double ncells = (double)s->dims[0] * s->dims[1] * s->dims[2];
    if (ncells >= 4294967295.0) { why = "too many grid cells (>= 2^32 - 1)"; return PSB_EINVAL; }
    if (s->method != PSB_WCSPH && s->method != PSB_PCISPH && s->method != PSB_DEM) { why = "unknown method"; return PSB_EINVAL; }
    if (s->method == PSB_DEM) {
        if (!(s->dem_spring >= 0) || !(s->dem_damping >= 0) || !std::isfinite(s->dem_shear) ||
            !std::isfinite(s->dem_attraction)) { why = "DEM: spring, damping must be >= 0"; return PSB_EINVAL; }
        if (s->profile == PSB_PROFILE_CONFIG && (!(s->particle_radius > 0) || s->h < 2.0 * s->particle_radius * (1.0 - 1e-6))) {
            why = "DEM config: particle_radius > 0 and h >= 2 particle_radius (contacts must be listed)";
            return PSB_EINVAL;
        }
        if (s->profile == PSB_PROFILE_CONFIG && (s->dem_shear != 0 || s->dem_attraction != 0)) {
            why = "DEM config: shear and attraction are reference-profile terms";
            return PSB_EINVAL;
        }
    }
    if (s->profile != PSB_PROFILE_REF && s->profile != PSB_PROFILE_CONFIG) { why = "unknown profile"; return PSB_EINVAL; }
    if (s->min_iters < 0 || s->max_iters < s->min_iters || s->max_iters > PSB_MAX_ITERS) {
        why = "need 0 <= min_iters <= max_iters <= PSB_MAX_ITERS";
        return PSB_EINVAL;
    }
    if (s->nbr_cap < 0 || s->nbr_cap > 4096) { why = "nbr_cap out of range"; return PSB_EINVAL; }
    if (s->warm_start != PSB_WARM_ZERO && s->warm_start != PSB_WARM_PREVIOUS && s->warm_start != PSB_WARM_LEARNED) {
        why = "unknown warm_start";
        return PSB_EINVAL;
    }
    {
        const double ws = s->spacing > 0 ? s->spacing : std::cbrt(s->mass / s->rho0);
        if (!(ws > 0)) { why = "spacing must be positive"; return PSB_EINVAL; }
        for (int a = 0; a < 3; ++a)
            if (!((double)s->box_max[a] - s->box_min[a] > 2.0 * s->h)) { why = "box narrower than 2h"; return PSB_EINVAL; }
    }
    if ((double)s->n_max * (s->nbr_cap ? s->nbr_cap : 128) >= 9.0e18) { why = "list too large"; return PSB_EINVAL; }
    return PSB_OK;
}

// Scene constants in FP64 on the host, then stored as FP32.
Params derive(const psb_scene& s) {
    Params P{};
    const double pi = 3.14159265358979323846;
    const double h = s.h, m = s.mass;
    P.g.gx = s.grid_min[0]; P.g.gy = s.grid_min[1]; P.g.gz = s.grid_min[2];
    P.g.cell = s.cell;
    P.g.nx = s.dims[0]; P.g.ny = s.dims[1]; P.g.nz = s.dims[2];
    P.cap = s.nbr_cap ? s.nbr_cap : 128;
    // list cut-off: the reference's h, or (1 + skin) h in the config profile
    const double hl = s.profile == PSB_PROFILE_CONFIG ? h * (1.0 + s.skin) : h;
    P.h = hl;
    // sqrt_rn is monotone, so {x >= 0 : sqrt_rn(x) <= h} is [0, X]: find X
    // from h*h by single ulps with the host's correctly rounded sqrt
    double X = hl * hl;
    while (std::sqrt(X) > hl) X = std::nextafter(X, 0.0);
    while (std::sqrt(std::nextafter(X, INFINITY)) <= hl) X = std::nextafter(X, INFINITY);
    P.h2_exact = X;
    const float h2f = (float)(hl * hl);
    P.h2_lo = h2f * (1.f - 1e-5f);
    P.h2_hi = h2f * (1.f + 1e-5f);
    P.h2 = h2f;
    P.inv_h = (float)(1.0 / h);
    P.inv_h2 = (float)(1.0 / (h * h));
    P.k_rho = (float)(315.0 * m / (64.0 * pi * h * h * h));
    const double G = 45.0 / (pi * h * h * h * h);
    P.k_grad = (float)(m * G);
    P.mass = (float)m;
    P.k_visc = (float)(s.mu * m * 45.0 / (pi * h * h * h * h * h));
    P.k_surf = (float)(945.0 * m / (32.0 * pi * h * h * h * h * h));
    P.ref = s.profile == PSB_PROFILE_REF;
    P.pci = s.method == PSB_PCISPH;
    // The reference's PCISPH kernel sets sigma = 0.0728 (PciSphSystem_Kernel.cu:161)
    P.sigma = (float)(P.pci ? 0.0728 : s.sigma);
    P.l = (float)s.l;
    P.surface = P.ref ? 1 : 0;
    const double dt = (double)s.dt;
    const double beta = 2.0 * (m * dt / s.rho0) * (m * dt / s.rho0);
    P.k_press = (float)(1.0 / (beta * G * G));
    P.rho0 = (float)s.rho0;
    P.rho0_d = s.rho0;
    P.eos_k = (float)(P.ref ? s.k : s.k * s.rho0 / 7.0);
    P.dt = s.dt;
    if (P.ref && P.pci) {            // forcesAccum = (0, -9.81 rho, 0), PciSphSystem_Kernel.cu:168
        P.gx = 0.f; P.gy = -9.81f; P.gz = 0.f;
    } else {
        P.gx = s.gravity[0]; P.gy = s.gravity[1]; P.gz = s.gravity[2];
    }
    P.wlo_x = s.box_min[0] + s.particle_radius; P.wlo_y = s.box_min[1] + s.particle_radius;
    P.wlo_z = s.box_min[2] + s.particle_radius;
    P.whi_x = s.box_max[0] - s.particle_radius; P.whi_y = s.box_max[1] - s.particle_radius;
    P.whi_z = s.box_max[2] - s.particle_radius;
    P.xsph_k = (float)(P.ref || !P.pci ? 0.0 : s.xsph * 315.0 * m / (64.0 * pi * h * h * h) / s.rho0);
    P.dem = s.method == PSB_DEM;
    if (P.dem) {
        P.pci = 0;
        P.dem_k = (float)s.dem_spring;
        P.dem_c = (float)s.dem_damping;
        P.dem_s = (float)s.dem_shear;
        P.dem_a = (float)s.dem_attraction;
        // REF: collideDist = (float)(h_A + h_B), contact while d < 2 collideDist
        P.dem_R = P.ref ? (float)(h + h) : (float)(2.0 * s.particle_radius);
        P.dem_range = P.ref ? 2.f * P.dem_R : P.dem_R;
        P.dem_mass = (float)m;
        P.dem_inv_mass = (float)(1.0 / m);
    }
    P.wall_k = (float)s.wall_k;     // config: penalty outside the faces (bx0..bz1)
    P.wall_c = (float)s.wall_c;
    P.bx0 = s.box_min[0]; P.by0 = s.box_min[1]; P.bz0 = s.box_min[2];
    P.bx1 = s.box_max[0]; P.by1 = s.box_max[1]; P.bz1 = s.box_max[2];
    const double ws = s.spacing > 0 ? s.spacing : std::cbrt(m / s.rho0);
    {   // Solenthaler & Pajarola 2009, sec. 4: delta from a particle with a filled neighbourhood
        const int R = (int)std::ceil(h / ws);
        double W1[3] = {0, 0, 0}, W2 = 0;
        for (int k = -R; k <= R; ++k)
            for (int j = -R; j <= R; ++j)
                for (int i = -R; i <= R; ++i) {
                    if (!i && !j && !k) continue;
                    const double r = ws * std::sqrt((double)(i * i + j * j + k * k));
                    if (r >= h) continue;
                    const double gw = G * (1.0 - r / h) * (1.0 - r / h);
                    W1[0] -= gw * i * ws / r; W1[1] -= gw * j * ws / r; W1[2] -= gw * k * ws / r;
                    W2 += gw * gw;
                }
        P.k_delta = (float)(1.0 / (beta * (W1[0] * W1[0] + W1[1] * W1[1] + W1[2] * W1[2] + W2)));
    }
    P.hf = (float)h;
    return P;
}

// ---- small device helpers: packing and id-order scatter -------------------

__global__ void k_pack3(int n, const float* __restrict__ src, float4* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src ? make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}
__global__ void k_pack3d(int n, const double* __restrict__ src, float4* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src ? make_float4(__double2float_rn(src[3 * i]), __double2float_rn(src[3 * i + 1]),
                                   __double2float_rn(src[3 * i + 2]), 0.f)
                     : make_float4(0.f, 0.f, 0.f, 0.f);
}
__global__ void k_init_ids(int n, const float* __restrict__ pres, int* __restrict__ ids, float2* __restrict__ rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { ids[i] = i; rp[i] = make_float2(0.f, pres ? pres[i] : 0.f); }
}
__global__ void k_iota(int n, int* __restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ids[i] = i;
}
__global__ void k_init_rp(int n, const float* __restrict__ pres, float2* __restrict__ rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rp[i] = make_float2(0.f, pres ? pres[i] : 0.f);
}
__global__ void k_scatter3(int n, const int* __restrict__ ids, const float4* __restrict__ src, float* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) { const int id = ids[t]; const float4 v = src[t]; dst[3 * id] = v.x; dst[3 * id + 1] = v.y; dst[3 * id + 2] = v.z; }
}
__global__ void k_scatter3d(int n, const int* __restrict__ ids, const float4* __restrict__ src, double* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) { const int id = ids[t]; const float4 v = src[t]; dst[3 * id] = v.x; dst[3 * id + 1] = v.y; dst[3 * id + 2] = v.z; }
}
__global__ void k_scatter_rp(int n, const int* __restrict__ ids, const float2* __restrict__ rp, int comp, float* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[ids[t]] = comp ? rp[t].y : rp[t].x;
}
__global__ void k_scatter_rows8(int n, const int* __restrict__ ids, const float* __restrict__ src, float* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float4* s = reinterpret_cast<const float4*>(src) + 2 * (size_t)t;
    float4* d = reinterpret_cast<float4*>(dst) + 2 * (size_t)ids[t];
    d[0] = s[0];
    d[1] = s[1];
}
__global__ void k_scatter_u32(int n, const int* __restrict__ ids, const uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[ids[t]] = src[t];
}

inline int blocks(int n) { return (n + psb::kBlock - 1) / psb::kBlock; }

int bits_for(size_t ncells) {
    int b = 1;
    while (b < 32 && ((size_t)1 << b) < ncells) ++b;
    return b;
}

// Whether the density pass at x is folded into the neighbour build
// (schedule 2): one config-profile PCISPH scene; batches, the reference
// profile, WCSPH and DEM run schedule 2 as schedule 0.
bool can_fuse_density(const psb_ctx* c, const Params& P) { return !c->batch && P.pci && !P.ref && !P.dem; }
bool fused_density(const psb_ctx* c, const Params& P) { return can_fuse_density(c, P) && P.tune.nbr_schedule == 2; }

// Grid, sort, reorder, neighbour lists, density at x. keep_p: leave the
// carried pressure in place even where the scene starts every step from 0.
int build(psb_ctx* c, bool keep_p = false, bool features = false) {
    cudaStream_t st = c->stream;
    Params P = c->P;
    P.n = c->n;
    const int n = c->n;
    const int rs = c->sorted >= 0 ? c->sorted : c->stale;       // cells occupied by the previous sort
    const int rn = c->sorted >= 0 ? c->sorted_n : c->stale_n;
    if (rs >= 0) timed(c, "reset_cells", [&] { psb::launch_reset_cells(st, rn, c->keys[rs], c->cell_start); });
    c->stale = -1;
    cudaMemsetAsync(c->flags, 0, 8 * sizeof(int), st);
    timed(c, "cell_keys", [&] {
        psb::launch_cell_keys(st, P, c->pos[c->cs], c->ids[c->cr], c->keys[0], c->vals[0], &c->flags[4]);
    });
    int res = 0;
    timed(c, "radix_sort", [&] { res = psb::radix_sort(st, n, c->key_bits, c->keys, c->vals, c->hist, c->hist_blocks); });
    const int os = c->cs, orr = c->cr, ns = os ^ 1, nr = orr ^ 1;
    // The first step after an upload gathers the positions first and the
    // rest of the state after its neighbour build, once the upload's copies
    // of it are in: they overlap the grid and the build. Other steps gather
    // everything in one launch.
    const bool split = capturing(st) ? c->capture_split : c->in_pending;
    if (split) {
        timed(c, "reorder_pos", [&] {
            psb::launch_reorder_pos(st, n, c->keys[res], c->vals[res], c->pos[os], c->ids[orr], c->pos[ns], c->ids[nr],
                                    c->cell_start, c->cell_end);
        });
    } else {
        timed(c, "reorder", [&] {
            psb::launch_reorder(st, n, c->keys[res], c->vals[res], c->pos[os], c->vel[os], c->vap[os], c->rp[orr],
                                c->ids[orr], c->pos[ns], c->vel[ns], c->vap[ns], c->rp[nr], c->ids[nr], c->cell_start,
                                c->cell_end);
        });
    }
    auto reorder_state = [&] {
        if (!split) return;
        wait_inputs(c, st);
        timed(c, "reorder_state", [&] {
            psb::launch_reorder_state(st, n, c->vals[res], c->vel[os], c->vap[os], c->rp[orr], c->vel[ns], c->vap[ns],
                                      c->rp[nr]);
        });
    };
    c->cs = ns;
    c->cr = nr;
    c->sorted = res;
    c->sorted_n = n;
    // boundary lists first: the density at x reads them
    if (c->bnd_n > 0)
        timed(c, "build_bnd_nbr", [&] {
            psb::launch_build_bnd_nbr(st, P, c->pos[c->cs], c->keys[res], c->bnd_cs, c->bnd_ce, c->bnd_count,
                                      c->bnd_list, c->flags);
        });
    const int zero_p = !keep_p && P.pci && (P.ref || c->sc.warm_start == PSB_WARM_ZERO);
    // the learned warm start and its data collection take their inputs from the density pass at x
    float* feats = features ? c->feats : nullptr;
    const int nfeat = psb::mlp_inputs(c->mlp_arch);
    if (fused_density(c, P)) {
        reorder_state();
        timed(c, "build_nbr", [&] {
            psb::launch_build_density(st, P, c->pos[c->cs], c->vel[c->cs], c->keys[res], c->cell_start, c->cell_end,
                                      c->nbr_count, c->nbr_list, c->flags, c->rp[c->cr], c->rho_x, zero_p, c->p_scale,
                                      feats, nfeat);
        });
    } else {
        timed(c, "build_nbr", [&] {
            psb::launch_build_nbr(st, P, c->pos[c->cs], c->keys[res], c->cell_start, c->cell_end, c->nbr_count,
                                  c->nbr_list, c->flags);
        });
        reorder_state();
        if (!P.dem)
            timed(c, "density_x", [&] {
                psb::launch_density_x(st, P, c->pos[c->cs], c->vel[c->cs], c->nbr_count, c->nbr_list, c->rp[c->cr],
                                      c->rho_x, zero_p, c->p_scale, feats, nfeat);
            });
    }
    c->built = true;
    return cuda_check(c, cudaGetLastError(), "launch");
}

int read_flags(psb_ctx* c) {
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_flags, c->flags, 8 * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "flags"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "sync"));
    c->stats.nbr_max = c->h_flags[1];
    long long tot;
    std::memcpy(&tot, &c->h_flags[2], 8);
    c->stats.nbr_total = tot;
    c->stats.clamped = c->h_flags[4];
    if (c->h_flags[0]) return fail(c, PSB_EOVERFLOW_NBR, "a particle has " + std::to_string(c->h_flags[1]) +
                                                             " neighbours, more than nbr_cap " + std::to_string(c->cap));
    return PSB_OK;
}

void release_graphs(psb_ctx* c);

// ---- the corrector loop on the device: batches and config-profile PCISPH ---

// A boundary moving with the corrector: its reaction at the committed
// pressures rp[r] (fluid at the start positions pos[s]) and its prediction.
void move_boundary(psb_ctx* c, cudaStream_t st, const Params& P, int s, int r) {
    timed(c, "bnd_move", [&] {
        psb::launch_bnd_move(st, P, c->bnd_n, c->pos[s], c->rp[r], c->cell_start, c->cell_end, c->bnd_vel, c->bnd_fext,
                             c->bnd_inv_mass, c->bnd_pred, c->bnd_react);
    });
}

// The corrector of a batch (or of one config-profile PCISPH scene, a batch
// of one): k_batch_begin, then {density pass, decision, pressure-force pass}
// until every scene has converged or max_iters passes have run. The predictions stay in xs[0]: the config profile's pressure-
// force pass reads the start positions, never x*, so it updates x* in place.
// capture: enqueue the loop as a while node of the graph being captured on
// the context's stream; else drive it from the host, one 4-byte read per pass.
int batch_corrector(psb_ctx* c, const Params& P, int s, int r, bool capture) {
    cudaStream_t st = c->stream;
    const int S = c->nscenes;
    const int max_it = c->sc.max_iters;
    const bool moving = P.bnd_pred != nullptr;
    // the persistent corrector has no pass that moves the boundary: a moving
    // boundary takes the per-pass launches
    if (c->corrector == PSB_CORRECTOR_PERSISTENT && max_it > 0 && !moving) {     // begins the loop itself
        cudaError_t e = cudaSuccess;
        timed(c, "corrector_persistent", [&] {
            e = psb::launch_corrector_persistent(st, P, c->pos[s], c->vap[s], c->fnp, c->xs[0], c->rp[r], c->rpc,
                                                 c->nbr_count, c->nbr_list, c->vs, S, c->sc.min_iters, max_it,
                                                 c->sc.eta, c->d_active, c->d_err_scene, c->d_err_sh, c->d_loop);
        });
        return cuda_check(c, e, "persistent corrector");
    }
    timed(c, "batch_begin", [&] {
        psb::launch_batch_begin(st, S, max_it, c->d_active, c->d_err_scene, c->d_err_sh, (PSB_MAX_ITERS + 1) * S,
                                c->d_loop);
    });
    if (max_it == 0) return PSB_OK;
    auto body = [&](cudaStream_t bs, cudaGraphConditionalHandle h, int set_handle) {
        timed(c, "pci_density", [&] {
            psb::launch_pci_density(bs, P, c->xs[0], c->rp[r], c->nbr_count, c->nbr_list, c->rpc,
                                    c->batch ? nullptr : c->d_err_scene);
        });
        timed(c, "batch_decide", [&] {
            psb::launch_batch_decide(bs, S, c->sc.min_iters, max_it, c->sc.eta, c->d_active, c->d_err_scene,
                                     c->d_err_sh, c->d_loop, h, set_handle);
        });
        timed(c, "pci_force_predict", [&] {
            psb::launch_pci_force_predict(bs, P, c->pos[s], c->vap[s], c->fnp, c->xs[1], c->rpc, c->nbr_count,
                                          c->nbr_list, c->xs[0], c->vs, c->rp[r]);
        });
        // the boundary predicted with the pressures the fluid's prediction
        // just used (once the scene has converged, the same pressures again)
        if (moving) move_boundary(c, bs, P, s, r);
    };
    if (!capture) {
        for (int k = 0; k < max_it; ++k) {
            body(st, 0, 0);
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_loop + 1, c->d_loop + 1, sizeof(int), cudaMemcpyDeviceToHost, st),
                               "loop"));
            PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "sync"));
            if (!c->h_loop[1]) break;
        }
        return PSB_OK;
    }
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    PSB_TRY(cuda_check(c, cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd), "capture info"));
    cudaGraphConditionalHandle h;
    PSB_TRY(cuda_check(c, cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault), "conditional handle"));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    PSB_TRY(cuda_check(c, cudaGraphAddNode(&node, g, deps, nd, &np), "while node"));
    cudaGraph_t body_graph = np.conditional.phGraph_out[0];
    PSB_TRY(cuda_check(c, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
                       "capture dependencies"));
    PSB_TRY(cuda_check(c, cudaStreamBeginCaptureToGraph(c->cap_stream, body_graph, nullptr, nullptr, 0,
                                                        cudaStreamCaptureModeThreadLocal), "body capture"));
    body(c->cap_stream, h, 1);
    cudaGraph_t ended = nullptr;
    return cuda_check(c, cudaStreamEndCapture(c->cap_stream, &ended), "body capture");
}

// One step of a batch, or of a single config-profile PCISPH scene, enqueued
// on the context's stream (or captured from it). A single scene's pressure-
// force pass reads the decision's active word and does nothing once the
// scene has converged, as a batch's retired scenes do.
int enqueue_loop_step(psb_ctx* c, bool capture) {
    const bool collect = c->collect_stride > 0;
    const int mode = c->sc.warm_start;
    PSB_TRY(build(c, mode != PSB_WARM_ZERO || collect, mode == PSB_WARM_LEARNED || collect));
    cudaStream_t st = c->stream;
    Params P = c->P;
    P.n = c->n;
    if (!c->batch) P.active = c->d_active;
    const int s = c->cs, r = c->cr;
    const bool moving = c->bnd_moving && c->bnd_n > 0;
    if (moving) P.bnd_pred = c->bnd_pred;
    if (mode == PSB_WARM_LEARNED) {
        timed(c, "mlp_infer", [&] {
            psb::launch_mlp_infer(st, c->mlp_arch, c->n, c->feats, c->mlp_wbf, c->p_scale, c->rp[r]);
        });
    } else if (mode == PSB_WARM_ZERO && collect) {
        psb::launch_zero_pressure(st, c->n, c->rp[r]);
    }
    timed(c, "pci_init", [&] {
        psb::launch_pci_init(st, P, c->pos[s], c->vel[s], c->vap[s], c->rp[r], c->nbr_count, c->nbr_list,
                             mode == PSB_WARM_ZERO ? 0 : 1, c->fnp, c->xs[0], c->vs);
    });
    if (moving) move_boundary(c, st, P, s, r);     // the boundary's first prediction, with the initial pressure
    PSB_TRY(batch_corrector(c, P, s, r, capture));
    const float4* v_commit = c->vs;
    if (P.xsph_k != 0.f) {
        timed(c, "xsph", [&] { psb::launch_xsph(st, P, c->xs[0], c->vs, c->nbr_count, c->nbr_list, c->xs[1]); });
        v_commit = c->xs[1];
    }
    timed(c, "pci_commit", [&] {
        psb::launch_pci_commit(st, P, c->xs[0], v_commit, c->rpc, c->sc.max_iters > 0, c->pos[s], c->vel[s], c->vap[s],
                               c->rp[r]);
    });
    return cuda_check(c, cudaGetLastError(), "launch");
}

// Captures the step from the current state parity into c->gexec[c->cs], on
// the context's own capture stream (nothing runs; the graph is launched on
// the caller's stream, which may be the legacy one).
int capture_loop_step(psb_ctx* c, int p) {
    c->capture_split = p >= 2;
    cudaStream_t user = c->stream;
    cudaStream_t st = c->cap_main;
    PSB_TRY(cuda_check(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture"));
    const int saved_cs = c->cs, saved_cr = c->cr, saved_sorted = c->sorted, saved_stale = c->stale;
    c->stream = st;
    const int rc = enqueue_loop_step(c, true);
    c->stream = user;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    // capturing ran none of it: the host state is the one before the step
    c->graph_sorted = c->sorted;
    c->cs = saved_cs; c->cr = saved_cr; c->sorted = saved_sorted; c->stale = saved_stale;
    if (rc != PSB_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc != PSB_OK ? rc : cuda_check(c, e, "capture");
    }
    const cudaError_t ei = cudaGraphInstantiate(&c->gexec[p], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) { c->gexec[p] = nullptr; return cuda_check(c, ei, "graph instantiate"); }
    c->graph_n = c->n;
    return PSB_OK;
}

int step_loop(psb_ctx* c, bool last) {
    cudaStream_t st = c->stream;
    const int S = c->nscenes;
    const bool collect = c->collect_stride > 0;
    // a graph holds the reset of the previous sort's cells: there must be one
    // (after an upload, the set before it), of the same size
    const int prev_n = c->sorted >= 0 ? c->sorted_n : (c->stale >= 0 ? c->stale_n : -1);
    const bool graph = c->graph_on && !collect && !c->prof.on && prev_n == c->n;
    if (graph) {
        if (c->graph_n != c->n) release_graphs(c);       // emissions changed the particle count
        const int gi = c->cs + (c->in_pending ? 2 : 0);
        if (!c->gexec[gi]) PSB_TRY(capture_loop_step(c, gi));
        PSB_TRY(cuda_check(c, cudaGraphLaunch(c->gexec[gi], st), "graph launch"));
        c->in_pending = false;        // the graph waits for the upload's copies itself
        // what build() records of the step it enqueues
        c->sorted = c->graph_sorted;
        c->sorted_n = c->n;
        c->stale = -1;
        c->cs ^= 1;
        c->cr ^= 1;
        c->built = true;
    } else {
        PSB_TRY(enqueue_loop_step(c, false));
    }
    c->stats.steps += 1;
    if (!last && !collect) return PSB_OK;
    // per-scene results of this step
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_loop, c->d_loop, sizeof(int) * (2 + 4 * (size_t)S), cudaMemcpyDeviceToHost,
                                          st), "loop"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_err_sh, c->d_err_sh, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1) * S,
                                          cudaMemcpyDeviceToHost, st), "err"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "sync"));
    int iters = 0, all_conv = 1;
    for (int k = 0; k < S; ++k) {
        iters = std::max(iters, c->h_loop[2 + k]);
        all_conv &= c->h_loop[2 + S + k];
    }
    c->stats.iters = iters;
    c->stats.converged = all_conv;
    if (!c->batch) c->stats.iters_total = c->iters_total_base + c->h_loop[2 + 2 * S];
    if (collect && all_conv) {
        const int stride = c->collect_stride;
        const int offset = (int)(c->collect_steps % stride);
        const int rows = offset < c->n ? (c->n - offset + stride - 1) / stride : 0;
        psb::launch_collect(st, c->n, stride, offset, c->ds_rows, c->ds_cap, c->feats, c->rp[c->cr], c->p_scale, c->ds_X,
                            c->ds_T);
        c->ds_rows += (uint64_t)rows;
        c->collect_steps += 1;
    }
    if (!last) return PSB_OK;
    PSB_TRY(read_flags(c));
    for (int i = 0; i <= PSB_MAX_ITERS; ++i) {
        double m = 0.0;
        for (int k = 0; k < S; ++k) {
            const unsigned long long e = c->h_err_sh[(size_t)i * S + k];
            if (e) m = std::max(m, psb::unorder_double(e));
        }
        c->stats.err[i] = m;
    }
    if (!all_conv) return fail(c, PSB_ENOCONV, "corrector loop reached max_iters above eta in a scene of the batch");
    return PSB_OK;
}

// The emissions due this step (Emitters::emitParticles before the
// neighbour search, PciSphSystem.cpp:155-160): all of them, or none when
// they exceed the capacity.
int run_emitters(psb_ctx* c) {
    int64_t need = 0;
    for (const auto& e : c->emitters)
        if (e.done < e.e.duration) need += e.per;
    if (need == 0) return PSB_OK;
    if ((int64_t)c->n + need > (int64_t)c->n_max)
        return fail(c, PSB_EINVAL, "emitters: " + std::to_string(need) + " particles due, " +
                                       std::to_string(c->n_max - c->n) + " free of the context's capacity");
    cudaStream_t st = c->stream;
    const int dem = c->P.dem ? 1 : 0;
    for (auto& e : c->emitters) {
        if (e.done >= e.e.duration) continue;
        const int n0 = c->n, k = (int)e.per;
        float4* pos = c->pos[c->cs] ;
        if (e.d_list)
            psb::launch_emit_list(st, n0, k, e.d_list, e.e.velocity, dem, pos, c->vel[c->cs], c->vap[c->cs],
                                  c->ids[c->cr], c->rp[c->cr]);
        else
            psb::launch_emit_random(st, n0, k, e.e.type, e.e.count, (unsigned)e.done, e.e.seed, e.e.v, e.d_faces,
                                    e.e.velocity, dem, pos, c->vel[c->cs], c->vap[c->cs], c->ids[c->cr],
                                    c->rp[c->cr]);
        if (c->P.ext_force) cudaMemsetAsync(c->ext_force + n0, 0, sizeof(float4) * (size_t)k, st);
        c->n += k;
        e.done += 1;
    }
    c->built = false;
    return cuda_check(c, cudaGetLastError(), "emitters");
}

int step_once(psb_ctx* c, bool last) {
    if (c->batch) return step_loop(c, last);
    if (!c->emitters.empty()) PSB_TRY(run_emitters(c));
    if (c->P.pci && !c->P.ref) return step_loop(c, last);     // config PCISPH: the corrector decides on the device
    const bool need_prev_p = !c->P.ref && c->P.pci && (c->sc.warm_start != PSB_WARM_ZERO || c->collect_stride > 0);
    const bool features = !c->P.ref && c->P.pci && (c->sc.warm_start == PSB_WARM_LEARNED || c->collect_stride > 0);
    PSB_TRY(build(c, need_prev_p, features));
    cudaStream_t st = c->stream;
    Params P = c->P;
    P.n = c->n;
    const int s = c->cs, r = c->cr;
    int iters = 0, converged = 1;
    cudaMemsetAsync(c->err_hist, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1), st);
    if (P.dem) {
        const int o = s ^ 1;
        P.slot_ids = c->ids[r];
        timed(c, "dem_step", [&] {
            psb::launch_dem_step(st, P, c->pos[s], c->vel[s], c->nbr_count, c->nbr_list, c->pos[o], c->vel[o], c->vap[o],
                                 c->fnp);
        });
        if (P.n_coll > 0)
            timed(c, "colliders", [&] {
                psb::launch_apply_colliders(st, P, c->pos[s], nullptr, c->pos[o], c->vel[o], c->vap[o]);
            });
        c->cs = o;
        c->stats.iters = 0;
        c->stats.converged = 1;
    } else if (!P.pci) {
        const int o = s ^ 1;
        timed(c, "wcsph_force", [&] {
            psb::launch_wcsph_force(st, P, c->pos[s], c->vel[s], c->vap[s], c->rp[r], c->nbr_count, c->nbr_list,
                                    c->pos[o], c->vel[o], c->vap[o], c->fnp);
        });
        if (P.n_coll > 0)
            timed(c, "colliders", [&] {
                psb::launch_apply_colliders(st, P, c->pos[s], c->vap[s], c->pos[o], c->vel[o], c->vap[o]);
            });
        c->cs = o;
        c->stats.iters = 0;
        c->stats.converged = 1;
    } else {
        // reference-profile PCISPH: exactly three corrections from p = 0
        // (PciSphSystem.cu:30-61), no host round trip
        timed(c, "pci_init", [&] {
            psb::launch_pci_init(st, P, c->pos[s], c->vel[s], c->vap[s], c->rp[r], c->nbr_count, c->nbr_list, 0,
                                 c->fnp, c->xs[0], c->vs);
        });
        constexpr int kRefIters = 3;
        int xi = 0;
        for (int k = 0; k < kRefIters; ++k) {
            timed(c, "pci_density", [&] {
                psb::launch_pci_density(st, P, c->xs[xi], c->rp[r], c->nbr_count, c->nbr_list, c->rpc, &c->err_hist[k]);
            });
            timed(c, "pci_force_predict", [&] {
                psb::launch_pci_force_predict(st, P, c->pos[s], c->vap[s], c->fnp, c->xs[xi], c->rpc, c->nbr_count,
                                              c->nbr_list, c->xs[xi ^ 1], c->vs, c->rp[r]);
            });
            xi ^= 1;
        }
        timed(c, "pci_commit", [&] {
            psb::launch_pci_commit(st, P, c->xs[xi], c->vs, c->rpc, 1, c->pos[s], c->vel[s], c->vap[s], c->rp[r]);
        });
        iters = kRefIters;
        c->stats.iters = iters;
        c->stats.converged = converged;
        if (last)
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_err, c->err_hist, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1),
                                                  cudaMemcpyDeviceToHost, st), "err"));
    }
    c->stats.steps += 1;
    c->stats.iters_total += iters;
    PSB_TRY(cuda_check(c, cudaGetLastError(), "launch"));
    if (last) {
        PSB_TRY(read_flags(c));
        for (int i = 0; i <= PSB_MAX_ITERS; ++i)
            c->stats.err[i] = (P.pci && c->h_err[i]) ? psb::unorder_double(c->h_err[i]) : 0.0;
    }
    return PSB_OK;
}

}  // namespace

extern "C" {

int32_t psb_abi_version(void) { return PSB_ABI_VERSION; }

const char* psb_status_string(int32_t status) {
    if (status < 0 || status > PSB_ESTATE) return "unknown status";
    return kStatus[status];
}

const char* psb_last_error(const psb_ctx* c) { return c ? c->err.c_str() : ""; }

}  // extern "C"

namespace {

// Context and device buffers for `scene` (validated) over `ncells` grid cells.
int create_impl(const psb_scene* scene, size_t ncells, psb_ctx** out) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        std::fprintf(stderr, "psb_create: no CUDA device\n");
        return PSB_ECUDA;
    }
    psb_ctx* c = new psb_ctx();
    c->sc = *scene;
    if (c->sc.nbr_cap == 0) c->sc.nbr_cap = 128;
    c->P = derive(c->sc);
    c->n_max = scene->n_max;
    c->cap = c->P.cap;
    c->ncells = ncells;
    c->key_bits = bits_for(c->ncells);
    c->hist_blocks = psb::radix_blocks(c->n_max);
    cudaGetDevice(&c->device);
    const size_t n = (size_t)c->n_max;
    int rc = PSB_OK;
    for (int i = 0; i < 2 && rc == PSB_OK; ++i) {
        rc = dalloc(c, &c->pos[i], n); if (rc) break;
        rc = dalloc(c, &c->vel[i], n); if (rc) break;
        rc = dalloc(c, &c->vap[i], n); if (rc) break;
        rc = dalloc(c, &c->rp[i], n); if (rc) break;
        rc = dalloc(c, &c->ids[i], n); if (rc) break;
        rc = dalloc(c, &c->keys[i], n); if (rc) break;
        rc = dalloc(c, &c->vals[i], n); if (rc) break;
        rc = dalloc(c, &c->xs[i], n); if (rc) break;
    }
    if (!rc) rc = dalloc(c, &c->hist, (size_t)256 * c->hist_blocks + 256);
    if (!rc) rc = dalloc(c, &c->cell_start, c->ncells);
    if (!rc) rc = dalloc(c, &c->cell_end, c->ncells);
    if (!rc) rc = dalloc(c, &c->nbr_count, n);
    if (!rc) rc = dalloc(c, &c->nbr_list, psb::nbr_list_ints(n, c->cap));
    if (!rc) rc = dalloc(c, &c->fnp, n);
    if (!rc) rc = dalloc(c, &c->vs, n);
    if (!rc) rc = dalloc(c, &c->rpc, n);
    if (!rc) rc = dalloc(c, &c->rho_x, n);
    if (!rc) rc = dalloc(c, &c->err_hist, PSB_MAX_ITERS + 1);
    if (!rc) rc = dalloc(c, &c->flags, 8);
    // uploads and downloads stage every array at once: 3 x 12 + 2 x 4 bytes
    if (!rc) rc = dalloc(c, (char**)&c->stage, n * 48);
    if (!rc) rc = dalloc(c, &c->feats, n * 8);
    if (!rc) rc = dalloc(c, &c->mlp_w, psb::kMlpParams);
    if (!rc) rc = dalloc(c, &c->mlp_m1, psb::kMlpParams);
    if (!rc) rc = dalloc(c, &c->mlp_m2, psb::kMlpParams);
    if (!rc) rc = dalloc(c, &c->mlp_grad, psb::kMlpParams);
    if (!rc) rc = dalloc(c, &c->mlp_part, psb::kMlpGradPartials);
    if (!rc) rc = dalloc(c, &c->mlp_loss, 1);
    if (!rc) rc = dalloc(c, (uint16_t**)&c->mlp_wbf, psb::kMlpParams);
    if (!rc && cudaMemset(c->mlp_w, 0, sizeof(float) * psb::kMlpParams) != cudaSuccess) rc = PSB_ECUDA;
    if (!rc && cudaMemset(c->mlp_wbf, 0, 2 * psb::kMlpParams) != cudaSuccess) rc = PSB_ECUDA;
    if (!rc && cudaMallocHost((void**)&c->h_err, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1)) != cudaSuccess) rc = PSB_ENOMEM;
    if (!rc && cudaMallocHost((void**)&c->h_flags, 8 * sizeof(int)) != cudaSuccess) rc = PSB_ENOMEM;
    if (!rc && cudaMemset(c->cell_start, 0xFF, sizeof(uint32_t) * c->ncells) != cudaSuccess) rc = PSB_ECUDA;
    if (!rc && cudaMemset(c->err_hist, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1)) != cudaSuccess) rc = PSB_ECUDA;
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = PSB_ECUDA;
    if (rc) {
        std::fprintf(stderr, "psb_create: %s\n", c->err.empty() ? "allocation failed" : c->err.c_str());
        cudaGetLastError();
        free_all(c);
        delete c;
        return rc;
    }
    std::memset(c->h_err, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1));
    {   // pressure scale of the learned warm start: rho0 |g| 0.1 m
        const double g = std::sqrt((double)scene->gravity[0] * scene->gravity[0] +
                                   (double)scene->gravity[1] * scene->gravity[1] +
                                   (double)scene->gravity[2] * scene->gravity[2]);
        c->p_scale = (float)(scene->rho0 * (g > 0 ? g : 9.81) * 0.1);
    }
    c->first = {0, (int64_t)scene->n_max};
    *out = c;
    return PSB_OK;
}

// The parameters every scene of a batch must share; returns the first that
// differs from scene 0, or nullptr.
const char* batch_mismatch(const psb_scene& a, const psb_scene& b) {
    if (a.h != b.h) return "h";
    if (a.mass != b.mass) return "mass";
    if (a.rho0 != b.rho0) return "rho0";
    if (a.k != b.k) return "k";
    if (a.mu != b.mu) return "mu";
    if (a.sigma != b.sigma || a.l != b.l) return "sigma/l";
    if (a.dt != b.dt) return "dt";
    for (int i = 0; i < 3; ++i)
        if (a.gravity[i] != b.gravity[i]) return "gravity";
    if (a.particle_radius != b.particle_radius) return "particle_radius";
    if (a.cell != b.cell) return "cell";
    if (a.profile != b.profile || a.method != b.method) return "profile/method";
    if (a.min_iters != b.min_iters || a.max_iters != b.max_iters || a.eta != b.eta) return "min_iters/max_iters/eta";
    if (a.wall_k != b.wall_k || a.wall_c != b.wall_c) return "wall_k/wall_c";
    if (a.nbr_cap != b.nbr_cap) return "nbr_cap";
    if (a.warm_start != b.warm_start) return "warm_start";
    if (a.spacing != b.spacing || a.skin != b.skin || a.xsph != b.xsph) return "spacing/skin/xsph";
    return nullptr;
}

// The device-side corrector's words for S scenes (batch.cu), their pinned
// mirrors, and the streams a CUDA-graph capture runs on.
int alloc_loop(psb_ctx* c, int S) {
    int rc = PSB_OK;
    if (!rc) rc = dalloc(c, &c->d_active, S);
    if (!rc) rc = dalloc(c, &c->d_err_scene, S);
    if (!rc) rc = dalloc(c, &c->d_err_sh, (size_t)(PSB_MAX_ITERS + 1) * S);
    if (!rc) rc = dalloc(c, &c->d_loop, 2 + 4 * (size_t)S);
    if (!rc && cudaMallocHost((void**)&c->h_loop, sizeof(int) * (2 + 4 * (size_t)S)) != cudaSuccess) rc = PSB_ENOMEM;
    if (!rc && cudaMallocHost((void**)&c->h_err_sh, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1) * S) != cudaSuccess)
        rc = PSB_ENOMEM;
    if (!rc) rc = cuda_check(c, cudaMemset(c->d_loop, 0, sizeof(int) * (2 + 4 * (size_t)S)), "loop");
    if (!rc) rc = cuda_check(c, cudaMemset(c->d_active, 1, S), "active");
    if (!rc) rc = cuda_check(c, cudaMemset(c->d_err_scene, 0, sizeof(unsigned long long) * S), "err");
    if (!rc) rc = cuda_check(c, cudaMemset(c->d_err_sh, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1) * S), "err");
    if (!rc) rc = cuda_check(c, cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking), "stream");
    if (!rc) rc = cuda_check(c, cudaStreamCreateWithFlags(&c->cap_main, cudaStreamNonBlocking), "stream");
    if (!rc) rc = cuda_check(c, cudaStreamCreateWithFlags(&c->copy_st, cudaStreamNonBlocking), "stream");
    if (!rc) rc = cuda_check(c, cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming), "event");
    if (!rc) rc = cuda_check(c, cudaEventCreateWithFlags(&c->ev_tail, cudaEventDisableTiming), "event");
    // a step's graph waits on ev_in: give it a first, completed record
    if (!rc) rc = cuda_check(c, cudaEventRecord(c->ev_in, c->copy_st), "event");
    if (!rc) {
        std::memset(c->h_loop, 0, sizeof(int) * (2 + 4 * (size_t)S));
        std::memset(c->h_err_sh, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1) * S);
    }
    return rc;
}

}  // namespace

extern "C" {

int psb_create(const psb_scene* scene, psb_ctx** out) {
    if (!out) return PSB_EINVAL;
    *out = nullptr;
    std::string why;
    if (validate(scene, why) != PSB_OK) {
        std::fprintf(stderr, "psb_create: %s\n", why.c_str());
        return PSB_EINVAL;
    }
    PSB_TRY(create_impl(scene, (size_t)scene->dims[0] * scene->dims[1] * scene->dims[2], out));
    psb_ctx* c = *out;
    if (const int rc = alloc_loop(c, 1)) {
        std::fprintf(stderr, "psb_create: %s\n", c->err.c_str());
        free_all(c);
        delete c;
        *out = nullptr;
        return rc;
    }
    return PSB_OK;
}

int psb_create_batch(const psb_scene* scenes, int32_t n_scenes, psb_ctx** out) {
    if (!out) return PSB_EINVAL;
    *out = nullptr;
    auto bad = [](const std::string& msg) {
        std::fprintf(stderr, "psb_create_batch: %s\n", msg.c_str());
        return PSB_EINVAL;
    };
    if (!scenes || n_scenes < 1 || n_scenes > 65535) return bad("need 1 <= n_scenes <= 65535 scenes");
    std::string why;
    int64_t total = 0;
    size_t cells = 0;
    for (int s = 0; s < n_scenes; ++s) {
        if (validate(&scenes[s], why) != PSB_OK) return bad("scene " + std::to_string(s) + ": " + why);
        if (const char* f = batch_mismatch(scenes[0], scenes[s]))
            return bad("scene " + std::to_string(s) + " differs from scene 0 in " + f);
        total += scenes[s].n_max;
        cells += (size_t)scenes[s].dims[0] * scenes[s].dims[1] * scenes[s].dims[2];
    }
    if (scenes[0].profile != PSB_PROFILE_CONFIG || scenes[0].method != PSB_PCISPH)
        return bad("batches are config-profile PCISPH scenes");
    if (total > 0x7fffffff) return bad("more than 2^31 - 1 particles in all");
    if ((double)cells >= 4294967295.0) return bad("too many grid cells in all (>= 2^32 - 1)");
    psb_scene u = scenes[0];
    u.n_max = (int32_t)total;
    psb_ctx* c = nullptr;
    PSB_TRY(create_impl(&u, cells, &c));
    const int S = n_scenes;
    c->batch = true;
    c->nscenes = S;
    c->first.assign(S + 1, 0);
    c->geom.resize(S);
    std::vector<uint16_t> slot_scene((size_t)total);
    uint32_t base = 0;
    for (int s = 0; s < S; ++s) {
        const psb_scene& sc = scenes[s];
        psb::SceneGeom& G = c->geom[s];
        G.bx0 = sc.box_min[0]; G.by0 = sc.box_min[1]; G.bz0 = sc.box_min[2];
        G.bx1 = sc.box_max[0]; G.by1 = sc.box_max[1]; G.bz1 = sc.box_max[2];
        // as derive() forms the single scene's bounds
        G.wlo_x = sc.box_min[0] + sc.particle_radius; G.wlo_y = sc.box_min[1] + sc.particle_radius;
        G.wlo_z = sc.box_min[2] + sc.particle_radius;
        G.whi_x = sc.box_max[0] - sc.particle_radius; G.whi_y = sc.box_max[1] - sc.particle_radius;
        G.whi_z = sc.box_max[2] - sc.particle_radius;
        G.g.gx = sc.grid_min[0]; G.g.gy = sc.grid_min[1]; G.g.gz = sc.grid_min[2];
        G.g.cell = sc.cell;
        G.g.nx = sc.dims[0]; G.g.ny = sc.dims[1]; G.g.nz = sc.dims[2];
        G.cell_base = base;
        base += (uint32_t)((size_t)sc.dims[0] * sc.dims[1] * sc.dims[2]);
        G.first = (int)c->first[s];
        G.count = sc.n_max;
        c->first[s + 1] = c->first[s] + sc.n_max;
        std::fill(slot_scene.begin() + c->first[s], slot_scene.begin() + c->first[s + 1], (uint16_t)s);
    }
    int rc = PSB_OK;
    if (!rc) rc = dalloc(c, &c->d_scenes, S);
    if (!rc) rc = dalloc(c, &c->d_slot_scene, (size_t)total);
    if (!rc) rc = cuda_check(c, cudaMemcpy(c->d_scenes, c->geom.data(), sizeof(psb::SceneGeom) * S, cudaMemcpyHostToDevice), "geom");
    if (!rc) rc = cuda_check(c, cudaMemcpy(c->d_slot_scene, slot_scene.data(), 2 * (size_t)total, cudaMemcpyHostToDevice), "slots");
    if (!rc) rc = alloc_loop(c, S);
    if (rc) {
        std::fprintf(stderr, "psb_create_batch: %s\n", c->err.c_str());
        free_all(c);
        delete c;
        return rc;
    }
    c->P.scenes = c->d_scenes;
    c->P.slot_scene = c->d_slot_scene;
    c->P.active = c->d_active;
    c->P.err_scene = c->d_err_scene;
    c->P.nscenes = S;
    *out = c;
    return PSB_OK;
}

int psb_destroy(psb_ctx* c) {
    if (!c) return PSB_EINVAL;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->copy_st) cudaStreamSynchronize(c->copy_st);
    free_all(c);
    delete c;
    return PSB_OK;
}

int psb_set_stream(psb_ctx* c, void* stream) {
    if (!c) return PSB_EINVAL;
    enter(c);
    c->prof.resolve(c->stream);
    const cudaStream_t next = (cudaStream_t)stream;
    if (next != c->stream) {
        // the new stream waits for the work already queued on the old one:
        // the context's buffers, and the pool memory that grow() frees in
        // stream order, may still be in use there
        cudaEvent_t done;
        PSB_TRY(cuda_check(c, cudaEventCreateWithFlags(&done, cudaEventDisableTiming), "psb_set_stream"));
        cudaError_t e = cudaEventRecord(done, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(next, done, 0);
        cudaEventDestroy(done);
        PSB_TRY(cuda_check(c, e, "psb_set_stream"));
    }
    c->stream = next;
    return PSB_OK;
}

static int size_bucket(int64_t n) {
    int b = 0;
    while (b < 62 && ((int64_t)1 << (b + 1)) <= n) ++b;
    return b;
}

// The launch configuration of the current particle count's bucket.
static void apply_tune(psb_ctx* c) {
    psb::Tune t{};
    auto it = c->tune_table.find(size_bucket(c->n));
    if (it != c->tune_table.end()) {
        const psb_tune& e = it->second;
        t = psb::Tune{e.nbr_block, e.nbr_schedule, e.density_block, e.init_block, e.pci_density_block, e.force_block,
                      e.xsph_block};
    }
    c->P.tune = t;
}

}  // extern "C"

namespace {
void release_graphs(psb_ctx* c) {
    cudaStreamSynchronize(c->stream);
    for (auto& g : c->gexec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}
}  // namespace

extern "C" {

static int upload_common(psb_ctx* c, int32_t n) {
    // forget the previous particle set; the next build clears its cells
    if (c->sorted >= 0) {
        c->stale = c->sorted;
        c->stale_n = c->sorted_n;
        c->sorted = -1;
    }
    c->n = n;
    c->cs = c->cr = 0;
    c->uploaded = true;
    c->built = false;
    apply_tune(c);
    if (!c->batch) c->iters_total_base = c->stats.iters_total;    // the loop words' sums restart at 0
    cudaMemsetAsync(c->d_loop, 0, sizeof(int) * (2 + 4 * (size_t)c->nscenes), c->stream);
    return PSB_OK;
}

int psb_upload(psb_ctx* c, int32_t n, const float* pos, const float* vel, const float* vel_half, const float* pressure) {
    if (!c || n <= 0 || n > c->n_max || !pos) return fail(c, PSB_EINVAL, "psb_upload: bad n or NULL pos");
    if (c->batch && n != c->n_max) return fail(c, PSB_EINVAL, "psb_upload: a batch takes all its scenes' particles");
    enter(c);
    upload_common(c, n);
    cudaStream_t st = c->stream, cp = c->copy_st;
    float* stage = (float*)c->stage;
    const size_t n3 = 3 * (size_t)n;
    // positions and ids on the context's stream: all that the next step's
    // grid and neighbour build read
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, pos, sizeof(float) * n3, cudaMemcpyHostToDevice, st), "upload"));
    k_pack3<<<blocks(n), psb::kBlock, 0, st>>>(n, stage, c->pos[0]);
    k_iota<<<blocks(n), psb::kBlock, 0, st>>>(n, c->ids[0]);
    // the rest on the copy stream, behind the positions' copy (and whatever
    // still reads the state buffers or the stage); the step gathers them
    // after its neighbour build, waiting on ev_in
    PSB_TRY(follow(c, st, cp));
    float* region = stage + n3;
    struct { const float* src; float4* dst; } parts[2] = {{vel, c->vel[0]}, {vel_half, c->vap[0]}};
    for (auto& p : parts) {
        if (p.src) PSB_TRY(cuda_check(c, cudaMemcpyAsync(region, p.src, sizeof(float) * n3, cudaMemcpyHostToDevice, cp), "upload"));
        k_pack3<<<blocks(n), psb::kBlock, 0, cp>>>(n, p.src ? region : nullptr, p.dst);
        region += n3;
    }
    if (pressure) PSB_TRY(cuda_check(c, cudaMemcpyAsync(region, pressure, sizeof(float) * n, cudaMemcpyHostToDevice, cp), "upload"));
    k_init_rp<<<blocks(n), psb::kBlock, 0, cp>>>(n, pressure ? region : nullptr, c->rp[0]);
    PSB_TRY(cuda_check(c, cudaEventRecord(c->ev_in, cp), "upload"));
    c->in_pending = true;
    return cuda_check(c, cudaGetLastError(), "upload");
}

int psb_upload_aos_f64(psb_ctx* c, int32_t n, const double* pos, const double* vel, const double* vel_half,
                       int32_t on_device) {
    if (!c || n <= 0 || n > c->n_max || !pos) return fail(c, PSB_EINVAL, "psb_upload_aos_f64: bad n or NULL pos");
    if (c->batch && n != c->n_max) return fail(c, PSB_EINVAL, "psb_upload_aos_f64: a batch takes all its scenes' particles");
    enter(c);
    upload_common(c, n);
    cudaStream_t st = c->stream;
    double* stage = (double*)c->stage;
    const size_t b3 = sizeof(double) * 3 * (size_t)n;
    struct { const double* src; float4* dst; } parts[3] = {{pos, c->pos[0]}, {vel, c->vel[0]}, {vel_half, c->vap[0]}};
    for (auto& p : parts) {
        const double* src = nullptr;
        if (p.src) {
            if (on_device) src = p.src;
            else {
                PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, p.src, b3, cudaMemcpyHostToDevice, st), "upload"));
                src = stage;
            }
        }
        k_pack3d<<<blocks(n), psb::kBlock, 0, st>>>(n, src, p.dst);
    }
    k_init_ids<<<blocks(n), psb::kBlock, 0, st>>>(n, nullptr, c->ids[0], c->rp[0]);
    return cuda_check(c, cudaGetLastError(), "upload");
}

int psb_download(psb_ctx* c, float* pos, float* vel, float* vel_half, float* density, float* pressure) {
    if (!c) return PSB_EINVAL;
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_download before psb_upload");
    enter(c);
    cudaStream_t st = c->stream, cp = c->copy_st;
    const int n = c->n;
    // each array is put in id order into a stage region of its own on the
    // context's stream and copied out on the copy stream, so the copy of
    // one overlaps the reordering of the next
    float* region = (float*)c->stage;
    struct { float* dst; const float4* src; } v3[3] = {{pos, c->pos[c->cs]}, {vel, c->vel[c->cs]}, {vel_half, c->vap[c->cs]}};
    for (auto& p : v3) {
        if (!p.dst) continue;
        k_scatter3<<<blocks(n), psb::kBlock, 0, st>>>(n, c->ids[c->cr], p.src, region);
        PSB_TRY(follow(c, st, cp));
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(p.dst, region, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, cp), "download"));
        region += 3 * (size_t)n;
    }
    struct { float* dst; int comp; } v1[2] = {{density, 0}, {pressure, 1}};
    for (auto& p : v1) {
        if (!p.dst) continue;
        k_scatter_rp<<<blocks(n), psb::kBlock, 0, st>>>(n, c->ids[c->cr], c->rp[c->cr], p.comp, region);
        PSB_TRY(follow(c, st, cp));
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(p.dst, region, sizeof(float) * n, cudaMemcpyDeviceToHost, cp), "download"));
        region += n;
    }
    PSB_TRY(cuda_check(c, cudaGetLastError(), "download"));
    // the context's stream also follows the copies (its next work may reuse the stage)
    PSB_TRY(follow(c, cp, st));
    return cuda_check(c, cudaStreamSynchronize(cp), "download");
}

int psb_download_aos_f64(psb_ctx* c, double* pos, double* vel, double* vel_half, int32_t on_device) {
    if (!c) return PSB_EINVAL;
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_download before psb_upload");
    enter(c);
    cudaStream_t st = c->stream;
    const int n = c->n;
    double* stage = (double*)c->stage;
    struct { double* dst; const float4* src; } v3[3] = {{pos, c->pos[c->cs]}, {vel, c->vel[c->cs]}, {vel_half, c->vap[c->cs]}};
    for (auto& p : v3) {
        if (!p.dst) continue;
        if (on_device) {
            k_scatter3d<<<blocks(n), psb::kBlock, 0, st>>>(n, c->ids[c->cr], p.src, p.dst);
        } else {
            k_scatter3d<<<blocks(n), psb::kBlock, 0, st>>>(n, c->ids[c->cr], p.src, stage);
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(p.dst, stage, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st), "download"));
        }
    }
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "download"));
    return cuda_check(c, cudaGetLastError(), "download");
}

int psb_step(psb_ctx* c, int32_t nsteps) {
    if (!c || nsteps < 0) return fail(c, PSB_EINVAL, "psb_step: bad argument");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_step before psb_upload");
    cudaSetDevice(c->device);
    // emitters write the state before the step's build, which otherwise
    // waits for the last upload's copies itself
    if (!c->emitters.empty()) join_inputs(c);
    int status = PSB_OK;
    for (int i = 0; i < nsteps; ++i) {
        const int rc = step_once(c, i == nsteps - 1);
        if (rc == PSB_ENOCONV) { status = rc; continue; }
        if (rc != PSB_OK) return rc;
    }
    if (c->prof.on) c->prof.resolve(c->stream);
    return status;
}

int psb_mlp_set_arch(psb_ctx* c, int32_t arch) {
    if (!c) return PSB_EINVAL;
    if (arch != PSB_MLP_SILU6 && arch != PSB_MLP_RELU7) return fail(c, PSB_EINVAL, "psb_mlp_set_arch: unknown network");
    enter(c);
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "arch"));
    c->mlp_arch = arch;
    c->mlp_set = false;          // the weights of the other network mean nothing here
    c->mlp_step = 0;
    PSB_TRY(cuda_check(c, cudaMemset(c->mlp_w, 0, sizeof(float) * psb::kMlpParams), "arch"));
    PSB_TRY(cuda_check(c, cudaMemset(c->mlp_wbf, 0, 2 * psb::kMlpParams), "arch"));
    release_graphs(c);
    return PSB_OK;
}

int psb_mlp_info(const psb_ctx* c, int32_t* arch, int32_t* n_inputs, int32_t* n_params) {
    if (!c) return PSB_EINVAL;
    if (arch) *arch = c->mlp_arch;
    if (n_inputs) *n_inputs = psb::mlp_inputs(c->mlp_arch);
    if (n_params) *n_params = psb::mlp_params(c->mlp_arch);
    return PSB_OK;
}

int psb_mlp_set_weights(psb_ctx* c, const float* w) {
    if (!c || !w) return PSB_EINVAL;
    enter(c);
    const int np = psb::mlp_params(c->mlp_arch);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->mlp_w, w, sizeof(float) * np, cudaMemcpyHostToDevice, c->stream), "weights"));
    cudaMemsetAsync(c->mlp_m1, 0, sizeof(float) * psb::kMlpParams, c->stream);
    cudaMemsetAsync(c->mlp_m2, 0, sizeof(float) * psb::kMlpParams, c->stream);
    psb::launch_to_bf16(c->stream, np, c->mlp_w, c->mlp_wbf);
    c->mlp_step = 0;
    c->mlp_set = true;
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "weights"));
    return cuda_check(c, cudaGetLastError(), "weights");
}

int psb_mlp_get_weights(psb_ctx* c, float* w) {
    if (!c || !w) return PSB_EINVAL;
    enter(c);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(w, c->mlp_w, sizeof(float) * psb::mlp_params(c->mlp_arch), cudaMemcpyDeviceToHost,
                                          c->stream), "weights"));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "weights");
}

int psb_mlp_collect(psb_ctx* c, int32_t stride, int64_t capacity) {
    if (!c || stride < 0 || (stride > 0 && capacity <= 0)) return fail(c, PSB_EINVAL, "psb_mlp_collect: bad argument");
    enter(c);
    c->collect_stride = stride;
    if (stride == 0) return PSB_OK;
    if ((uint64_t)capacity != c->ds_cap) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->ds_X);
        cudaFree(c->ds_T);
        c->ds_X = c->ds_T = nullptr;
        c->ds_cap = 0;
        PSB_TRY(dalloc(c, &c->ds_X, (size_t)capacity * 8));
        PSB_TRY(dalloc(c, &c->ds_T, (size_t)capacity));
        c->ds_cap = (uint64_t)capacity;
        c->ds_rows = 0;
    }
    return PSB_OK;
}

int psb_mlp_dataset(psb_ctx* c, int64_t* rows, float* X, float* T) {
    if (!c || !rows) return PSB_EINVAL;
    enter(c);
    const uint64_t r = c->ds_rows < c->ds_cap ? c->ds_rows : c->ds_cap;
    *rows = (int64_t)r;
    if (X && r) PSB_TRY(cuda_check(c, cudaMemcpyAsync(X, c->ds_X, sizeof(float) * 8 * r, cudaMemcpyDeviceToHost, c->stream), "dataset"));
    if (T && r) PSB_TRY(cuda_check(c, cudaMemcpyAsync(T, c->ds_T, sizeof(float) * r, cudaMemcpyDeviceToHost, c->stream), "dataset"));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "dataset");
}

int psb_mlp_train(psb_ctx* c, int32_t iters, int32_t batch, float lr, uint64_t seed, float* loss) {
    if (!c || iters < 0 || batch <= 0 || !(lr > 0)) return fail(c, PSB_EINVAL, "psb_mlp_train: bad argument");
    const uint64_t rows = c->ds_rows < c->ds_cap ? c->ds_rows : c->ds_cap;
    if (rows == 0) return fail(c, PSB_ESTATE, "psb_mlp_train: no recorded data");
    if (!c->mlp_set) return fail(c, PSB_ESTATE, "psb_mlp_train: set initial weights first");
    enter(c);
    cudaStream_t st = c->stream;
    if (batch > c->sel_cap) {
        cudaStreamSynchronize(st);
        cudaFree(c->sel);
        c->sel = nullptr;
        c->sel_cap = 0;
        PSB_TRY(dalloc(c, &c->sel, (size_t)batch));
        c->sel_cap = batch;
    }
    for (int it = 0; it < iters; ++it) {
        psb::launch_mlp_sample(st, batch, rows, seed + 0x100000001ull * (uint64_t)(c->mlp_step + 1), c->sel);
        timed(c, "mlp_train", [&] {
            psb::launch_mlp_grad(st, c->mlp_arch, batch, c->ds_X, c->ds_T, c->sel, c->mlp_wbf, c->mlp_part, c->mlp_grad,
                                 c->mlp_loss);
        });
        ++c->mlp_step;
        psb::launch_adam(st, psb::mlp_params(c->mlp_arch), c->mlp_w, c->mlp_grad, c->mlp_m1, c->mlp_m2, c->mlp_wbf, lr,
                         c->mlp_step);
    }
    if (loss) {
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(loss, c->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, st), "loss"));
    }
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "train"));
    return cuda_check(c, cudaGetLastError(), "train");
}

static int mlp_host_call(psb_ctx* c, const float* X, const float* T, int32_t n, float* y, float* loss, float* grad) {
    if (!c || !X || n <= 0) return fail(c, PSB_EINVAL, "psb_mlp: bad argument");
    enter(c);
    cudaStream_t st = c->stream;
    float *dX = nullptr, *dT = nullptr, *dy = nullptr;
    int rc = dalloc(c, &dX, (size_t)n * 8);
    if (!rc) rc = dalloc(c, &dT, (size_t)n);
    if (!rc) rc = dalloc(c, &dy, (size_t)n);
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(dX, X, sizeof(float) * 8 * n, cudaMemcpyHostToDevice, st), "mlp");
    if (!rc && T) rc = cuda_check(c, cudaMemcpyAsync(dT, T, sizeof(float) * n, cudaMemcpyHostToDevice, st), "mlp");
    if (!rc && y) {
        psb::launch_mlp_forward(st, c->mlp_arch, n, dX, c->mlp_wbf, dy);
        rc = cuda_check(c, cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, st), "mlp");
    }
    if (!rc && grad) {
        psb::launch_mlp_grad(st, c->mlp_arch, n, dX, dT, nullptr, c->mlp_wbf, c->mlp_part, c->mlp_grad, c->mlp_loss);
        rc = cuda_check(c, cudaMemcpyAsync(grad, c->mlp_grad, sizeof(float) * psb::mlp_params(c->mlp_arch),
                                           cudaMemcpyDeviceToHost, st), "mlp");
        if (!rc && loss) rc = cuda_check(c, cudaMemcpyAsync(loss, c->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, st), "mlp");
    }
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(st), "mlp");
    if (!rc) rc = cuda_check(c, cudaGetLastError(), "mlp");
    cudaFree(dX);
    cudaFree(dT);
    cudaFree(dy);
    return rc;
}

int psb_mlp_forward(psb_ctx* c, const float* X, int32_t n, float* y) {
    if (!y) return PSB_EINVAL;
    return mlp_host_call(c, X, nullptr, n, y, nullptr, nullptr);
}

int psb_mlp_loss_grad(psb_ctx* c, const float* X, const float* T, int32_t n, float* loss, float* grad) {
    if (!T || !grad) return PSB_EINVAL;
    return mlp_host_call(c, X, T, n, nullptr, loss, grad);
}

int psb_presolve(psb_ctx* c, int32_t iters) {
    if (!c || iters < 0) return fail(c, PSB_EINVAL, "psb_presolve: bad argument");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_presolve before psb_upload");
    if (!c->P.pci || c->P.ref) return fail(c, PSB_EINVAL, "psb_presolve: config-profile PCISPH scenes only");
    enter(c);
    PSB_TRY(build(c, /*keep_p=*/true));
    cudaStream_t st = c->stream;
    Params P = c->P;
    P.n = c->n;
    const int s = c->cs, r = c->cr;
    cudaMemsetAsync(c->err_hist, 0, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1), st);
    if (c->batch) cudaMemsetAsync(c->d_active, 1, c->nscenes, st);     // every scene takes every pass
    timed(c, "pci_init", [&] {
        psb::launch_pci_init(st, P, c->pos[s], c->vel[s], c->vap[s], c->rp[r], c->nbr_count, c->nbr_list, 1, c->fnp,
                             c->xs[0], c->vs);
    });
    int xi = 0;
    for (int k = 0; k < iters; ++k) {
        timed(c, "pci_density", [&] {
            psb::launch_pci_density(st, P, c->xs[xi], c->rp[r], c->nbr_count, c->nbr_list, c->rpc,
                                    &c->err_hist[k < PSB_MAX_ITERS ? k : PSB_MAX_ITERS]);
        });
        timed(c, "pci_force_predict", [&] {
            psb::launch_pci_force_predict(st, P, c->pos[s], c->vap[s], c->fnp, c->xs[xi], c->rpc, c->nbr_count,
                                          c->nbr_list, c->xs[xi ^ 1], c->vs, c->rp[r]);
        });
        xi ^= 1;
    }
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_err, c->err_hist, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1),
                                          cudaMemcpyDeviceToHost, st), "err"));
    PSB_TRY(read_flags(c));
    for (int i = 0; i <= PSB_MAX_ITERS; ++i) c->stats.err[i] = c->h_err[i] ? psb::unorder_double(c->h_err[i]) : 0.0;
    c->stats.iters = iters;
    return PSB_OK;
}

int psb_build_neighbors(psb_ctx* c) {
    if (!c) return PSB_EINVAL;
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_build_neighbors before psb_upload");
    enter(c);
    PSB_TRY(build(c));
    return read_flags(c);
}

int psb_warm_start(psb_ctx* c, float* features, float* pressure) {
    if (!c) return PSB_EINVAL;
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_warm_start before psb_upload");
    if (c->batch || !c->P.pci || c->P.ref)
        return fail(c, PSB_EINVAL, "psb_warm_start: single config-profile PCISPH scenes only");
    enter(c);
    const int mode = c->sc.warm_start;
    if (mode == PSB_WARM_LEARNED && !c->mlp_set) return fail(c, PSB_ESTATE, "psb_warm_start: no network weights set");
    PSB_TRY(build(c, /*keep_p=*/true, /*features=*/true));
    cudaStream_t st = c->stream;
    const int n = c->n;
    const int* ids = c->ids[c->cr];
    float* stage = (float*)c->stage;
    if (features) {
        k_scatter_rows8<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, c->feats, stage);
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(features, stage, sizeof(float) * 8 * (size_t)n, cudaMemcpyDeviceToHost, st),
                           "warm_start"));
        PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "warm_start"));
    }
    if (pressure) {
        if (mode == PSB_WARM_ZERO) {
            std::memset(pressure, 0, sizeof(float) * (size_t)n);
        } else {
            // the learned guess goes to the corrector's scratch: the carried
            // pressure, an input of the next step, stays in place
            const float2* src = c->rp[c->cr];
            if (mode == PSB_WARM_LEARNED) {
                psb::launch_mlp_infer(st, c->mlp_arch, n, c->feats, c->mlp_wbf, c->p_scale, c->rpc);
                src = c->rpc;
            }
            k_scatter_rp<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, src, 1, stage);
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(pressure, stage, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st),
                               "warm_start"));
        }
    }
    PSB_TRY(cuda_check(c, cudaGetLastError(), "warm_start"));
    return read_flags(c);
}

}  // extern "C"

namespace {

template <typename T>
int grow(psb_ctx* c, T** p, long long* cap, long long need) {
    if (need <= *cap) return PSB_OK;
    // Geometric growth, from the context's stream-ordered pool: outputs
    // such as a mesh grow a little with every call, and a cudaFree /
    // cudaMalloc pair waits for the whole device -- on a 4M-particle context
    // with its step graphs it measured 25-750 ms, against 4.4 ms for the
    // extraction it served.
    const long long alloc = std::max(need, *cap + *cap / 2);
    if (!c->pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = c->device;
        if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
            cudaGetLastError();
            c->pool = nullptr;
            return fail(c, PSB_ECUDA, "cudaMemPoolCreate failed");
        }
        uint64_t keep = UINT64_MAX;      // never hand freed memory back between growths
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (*p) cudaFreeAsync(*p, c->stream);
    *p = nullptr;
    *cap = 0;
    if (cudaMallocFromPoolAsync((void**)p, sizeof(T) * (size_t)alloc, c->pool, c->stream) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(c, PSB_ENOMEM, "allocation of " + std::to_string(sizeof(T) * (size_t)alloc) + " bytes failed");
    }
    *cap = alloc;
    return PSB_OK;
}

// Iso field of `g` into c->iso at the current positions (grid rebuilt first).
int iso_on_device(psb_ctx* c, const psb_iso_grid* g, double level, psb::IsoParams& Q) {
    if (!g) return fail(c, PSB_EINVAL, "iso grid is NULL");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "iso field before psb_upload");
    if (c->P.dem) return fail(c, PSB_EINVAL, "iso field: SPH scenes only");
    if (c->batch) return fail(c, PSB_EINVAL, "iso field: single-scene contexts only");
    long long nn = 1;
    for (int a = 0; a < 3; ++a) {
        if (g->dims[a] < 2 || !(g->spacing[a] > 0) || !std::isfinite(g->spacing[a]) || !std::isfinite(g->origin[a]))
            return fail(c, PSB_EINVAL, "iso grid: dims >= 2, finite spacing > 0, finite origin");
        nn *= g->dims[a];
    }
    if (3 * nn + 1 >= (1LL << 30)) return fail(c, PSB_EINVAL, "iso grid: at most 2^30 / 3 nodes");
    Q = psb::IsoParams{};
    for (int a = 0; a < 3; ++a) {
        Q.origin[a] = g->origin[a];
        Q.spacing[a] = g->spacing[a];
        Q.dims[a] = g->dims[a];
    }
    Q.level = level;
    const double h = c->sc.h;
    // Every node's particle-grid cell, widened by its ring, must fit the
    // device's int cell coordinates, and the reference profile's ring
    // floor(1 / scale) stays at 16 cells or fewer (the reference uses 0.65,
    // one ring), so each node's walk is bounded.
    const double corner[3] = {c->P.g.gx, c->P.g.gy, c->P.g.gz};
    for (int a = 0; a < 3; ++a) {
        const double lo = (g->origin[a] - corner[a]) / c->P.g.cell;
        const double hi = (g->origin[a] + (g->dims[a] - 1) * g->spacing[a] - corner[a]) / c->P.g.cell;
        if (!(std::fabs(lo) < 1073741824.0 && std::fabs(hi) < 1073741824.0))
            return fail(c, PSB_EINVAL, "iso grid: nodes lie too far from the particle grid");
    }
    if (c->P.ref) {
        if (!(g->scale >= 0.0625 && std::isfinite(g->scale)))
            return fail(c, PSB_EINVAL, "iso grid: reference profile needs a finite scale >= 1/16");
        Q.r = h / g->scale;
        Q.ring = (int)std::floor(1.0 / g->scale);
    } else {
        Q.ring = 1;      // cell >= h
        Q.inv_r2 = 1.0 / (h * h);
        Q.k_colour = 315.0 * c->sc.mass / (64.0 * 3.14159265358979323846 * h * h * h);
    }
    enter(c);
    PSB_TRY(build(c, /*keep_p=*/true));
    PSB_TRY(grow(c, &c->iso, &c->iso_cap, nn));
    Params P = c->P;
    P.n = c->n;
    timed(c, "iso_field", [&] {
        psb::launch_iso_field(c->stream, Q, P, c->pos[c->cs], c->rp[c->cr], c->cell_start, c->cell_end, c->iso);
    });
    return cuda_check(c, cudaGetLastError(), "iso field");
}

}  // namespace

extern "C" {

int psb_set_boundary(psb_ctx* c, int32_t n_bnd, const float* pos) {
    if (!c || n_bnd < 0 || (n_bnd > 0 && !pos)) return fail(c, PSB_EINVAL, "psb_set_boundary: bad argument");
    if (n_bnd > 0 && (c->P.ref || c->P.dem || c->batch))
        return fail(c, PSB_EINVAL, "psb_set_boundary: config-profile SPH, single-scene contexts only");
    enter(c);
    cudaStream_t st = c->stream;
    release_graphs(c);
    if (c->bnd_n > 0) {      // forget the previous set: clear its cells
        psb::launch_reset_cells(st, c->bnd_n, c->bnd_keys[c->bnd_res], c->bnd_cs);
        c->bnd_n = 0;
    }
    c->P.bnd = nullptr;
    c->P.bnd_count = nullptr;
    c->P.bnd_list = nullptr;
    c->bnd_moving = false;      // a new set is static until psb_set_boundary_motion
    if (n_bnd == 0) return cuda_check(c, cudaGetLastError(), "psb_set_boundary");
    const size_t nb = (size_t)n_bnd;
    if (!c->bnd_cs) {
        PSB_TRY(dalloc(c, &c->bnd_cs, c->ncells));
        PSB_TRY(dalloc(c, &c->bnd_ce, c->ncells));
        PSB_TRY(cuda_check(c, cudaMemset(c->bnd_cs, 0xFF, sizeof(uint32_t) * c->ncells), "boundary"));
        PSB_TRY(dalloc(c, &c->bnd_count, (size_t)c->n_max));
        PSB_TRY(dalloc(c, &c->bnd_list, psb::nbr_list_ints((size_t)c->n_max, psb_ctx::kBndCap)));
    }
    if ((long long)nb > c->bnd_cap_alloc) {
        cudaStreamSynchronize(st);
        cudaFree(c->bnd_raw); cudaFree(c->bnd_sorted); cudaFree(c->bnd_ids); cudaFree(c->bnd_iota); cudaFree(c->bnd_w);
        for (int i = 0; i < 2; ++i) { cudaFree(c->bnd_keys[i]); cudaFree(c->bnd_vals[i]); }
        cudaFree(c->bnd_hist);
        c->bnd_cap_alloc = 0;
        PSB_TRY(dalloc(c, &c->bnd_raw, nb));
        PSB_TRY(dalloc(c, &c->bnd_sorted, nb));
        PSB_TRY(dalloc(c, &c->bnd_ids, nb));
        PSB_TRY(dalloc(c, &c->bnd_iota, nb));
        PSB_TRY(dalloc(c, &c->bnd_w, nb));
        for (int i = 0; i < 2; ++i) {
            PSB_TRY(dalloc(c, &c->bnd_keys[i], nb));
            PSB_TRY(dalloc(c, &c->bnd_vals[i], nb));
        }
        PSB_TRY(dalloc(c, &c->bnd_hist, (size_t)256 * psb::radix_blocks((int)nb) + 256));
        c->bnd_cap_alloc = (long long)nb;
    }
    // positions through the staging buffer (n_max x 32 B), in chunks
    float* stage = (float*)c->stage;
    const size_t chunk = ((size_t)c->n_max * 32) / (3 * sizeof(float));
    for (size_t off = 0; off < nb; off += chunk) {
        const size_t m = std::min(chunk, nb - off);
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, pos + 3 * off, sizeof(float) * 3 * m, cudaMemcpyHostToDevice, st),
                           "boundary"));
        k_pack3<<<blocks((int)m), psb::kBlock, 0, st>>>((int)m, stage, c->bnd_raw + off);
    }
    cudaMemsetAsync(c->flags, 0, 8 * sizeof(int), st);
    c->bnd_res = psb::launch_bnd_prepare(st, c->P, n_bnd, c->bnd_raw, c->bnd_iota, c->bnd_keys, c->bnd_vals,
                                         c->bnd_hist, psb::radix_blocks(n_bnd), c->key_bits, c->bnd_sorted, c->bnd_ids,
                                         c->bnd_w, c->bnd_cs, c->bnd_ce, &c->flags[4]);
    // the bounding box, grown by the list cut-off
    float lo[3] = {pos[0], pos[1], pos[2]}, hi[3] = {pos[0], pos[1], pos[2]};
    for (size_t i = 1; i < nb; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], pos[3 * i + a]);
            hi[a] = std::max(hi[a], pos[3 * i + a]);
        }
    const float grow_by = (float)(c->P.h * 1.001) + 1e-6f;
    for (int a = 0; a < 3; ++a) { c->P.bnd_lo[a] = lo[a] - grow_by; c->P.bnd_hi[a] = hi[a] + grow_by; }
    c->bnd_n = n_bnd;
    c->P.bnd = c->bnd_sorted;
    c->P.bnd_count = c->bnd_count;
    c->P.bnd_list = c->bnd_list;
    c->P.bnd_cap = psb_ctx::kBndCap;
    c->built = false;
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_flags, c->flags, 8 * sizeof(int), cudaMemcpyDeviceToHost, st), "boundary"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "boundary"));
    if (c->h_flags[4]) return fail(c, PSB_EINVAL, "psb_set_boundary: boundary particles outside the grid");
    return cuda_check(c, cudaGetLastError(), "psb_set_boundary");
}

int psb_boundary_forces(psb_ctx* c, float* force) {
    if (!c || !force) return PSB_EINVAL;
    if (c->bnd_n == 0) return fail(c, PSB_ESTATE, "psb_boundary_forces: no boundary set");
    if (!c->built) return fail(c, PSB_ESTATE, "psb_boundary_forces: take a step first");
    enter(c);
    cudaStream_t st = c->stream;
    PSB_TRY(grow(c, &c->bnd_force, &c->bnd_force_cap, (long long)c->bnd_n));
    Params P = c->P;
    P.n = c->n;
    if (c->bnd_moving)      // the reaction the boundary's last prediction used
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->bnd_force, c->bnd_react, sizeof(float4) * (size_t)c->bnd_n,
                                              cudaMemcpyDeviceToDevice, st), "boundary forces"));
    else
        psb::launch_bnd_reaction(st, P, c->bnd_n, c->pos[c->cs], c->rp[c->cr], c->cell_start, c->cell_end,
                                 c->bnd_force);
    std::vector<float4> f((size_t)c->bnd_n);
    std::vector<int> ids((size_t)c->bnd_n);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(f.data(), c->bnd_force, sizeof(float4) * f.size(), cudaMemcpyDeviceToHost, st),
                       "boundary forces"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(ids.data(), c->bnd_ids, sizeof(int) * ids.size(), cudaMemcpyDeviceToHost, st),
                       "boundary forces"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "boundary forces"));
    for (int t = 0; t < c->bnd_n; ++t) {
        float* o = force + 3 * (size_t)ids[t];
        o[0] = f[t].x; o[1] = f[t].y; o[2] = f[t].z;
    }
    return cuda_check(c, cudaGetLastError(), "boundary forces");
}

int psb_set_boundary_motion(psb_ctx* c, const float* vel, const float* force, float mass) {
    if (!c) return PSB_EINVAL;
    enter(c);
    release_graphs(c);
    if (!vel) {
        c->bnd_moving = false;
        return PSB_OK;
    }
    if (!force || !(mass > 0.f) || !std::isfinite(mass))
        return fail(c, PSB_EINVAL, "psb_set_boundary_motion: bad argument");
    if (c->bnd_n == 0) return fail(c, PSB_ESTATE, "psb_set_boundary_motion: set the boundary first");
    if (c->batch || !c->P.pci || c->P.ref || c->P.dem)
        return fail(c, PSB_EINVAL, "psb_set_boundary_motion: config-profile PCISPH, single-scene contexts only");
    cudaStream_t st = c->stream;
    const int nb = c->bnd_n;
    long long cap = c->bnd_motion_cap;
    PSB_TRY(grow(c, &c->bnd_vel, &cap, (long long)nb));
    cap = c->bnd_motion_cap;
    PSB_TRY(grow(c, &c->bnd_fext, &cap, (long long)nb));
    cap = c->bnd_motion_cap;
    PSB_TRY(grow(c, &c->bnd_pred, &cap, (long long)nb));
    cap = c->bnd_motion_cap;
    PSB_TRY(grow(c, &c->bnd_react, &cap, (long long)nb));
    c->bnd_motion_cap = cap;
    // each array through the staging buffer into bnd_raw (input order),
    // then into sorted boundary slots
    float* stage = (float*)c->stage;
    const size_t chunk = ((size_t)c->n_max * 32) / (3 * sizeof(float));
    const float* src[2] = {vel, force};
    float4* dst[2] = {c->bnd_vel, c->bnd_fext};
    for (int a = 0; a < 2; ++a) {
        for (size_t off = 0; off < (size_t)nb; off += chunk) {
            const size_t m = std::min(chunk, (size_t)nb - off);
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, src[a] + 3 * off, sizeof(float) * 3 * m, cudaMemcpyHostToDevice,
                                                  st), "boundary motion"));
            k_pack3<<<blocks((int)m), psb::kBlock, 0, st>>>((int)m, stage, c->bnd_pred + off);
        }
        psb::launch_bnd_gather4(st, nb, c->bnd_ids, c->bnd_pred, dst[a]);
    }
    c->bnd_inv_mass = 1.f / mass;
    c->bnd_moving = true;
    return cuda_check(c, cudaGetLastError(), "psb_set_boundary_motion");
}

int psb_dem_forces(psb_ctx* c, float* force) {
    if (!c || !force) return PSB_EINVAL;
    if (!c->P.dem) return fail(c, PSB_EINVAL, "psb_dem_forces: DEM contexts only");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_dem_forces before psb_upload");
    enter(c);
    cudaStream_t st = c->stream;
    PSB_TRY(build(c));
    Params P = c->P;
    P.n = c->n;
    psb::launch_dem_forces(st, P, c->pos[c->cs], c->vel[c->cs], c->nbr_count, c->nbr_list, c->fnp);
    PSB_TRY(read_flags(c));
    std::vector<float4> f((size_t)c->n);
    std::vector<int> ids((size_t)c->n);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(f.data(), c->fnp, sizeof(float4) * f.size(), cudaMemcpyDeviceToHost, st),
                       "dem forces"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(ids.data(), c->ids[c->cr], sizeof(int) * ids.size(), cudaMemcpyDeviceToHost,
                                          st), "dem forces"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "dem forces"));
    for (int t = 0; t < c->n; ++t) {
        float* o = force + 3 * (size_t)ids[t];
        o[0] = f[t].x; o[1] = f[t].y; o[2] = f[t].z;
    }
    return cuda_check(c, cudaGetLastError(), "dem forces");
}

int psb_set_external_force(psb_ctx* c, const float* force) {
    if (!c) return PSB_EINVAL;
    if (!c->P.dem) return fail(c, PSB_EINVAL, "psb_set_external_force: DEM contexts only");
    enter(c);
    release_graphs(c);
    if (!force) {
        c->P.ext_force = nullptr;
        return PSB_OK;
    }
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_set_external_force before psb_upload");
    cudaStream_t st = c->stream;
    if (!c->ext_force) PSB_TRY(dalloc(c, &c->ext_force, (size_t)c->n_max));
    float* stage = (float*)c->stage;
    const int n = c->n;
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, force, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st),
                       "external force"));
    k_pack3<<<blocks(n), psb::kBlock, 0, st>>>(n, stage, c->ext_force);
    c->P.ext_force = c->ext_force;
    return cuda_check(c, cudaGetLastError(), "external force");
}

namespace {

// Why an object cannot be taken, or "".
std::string collider_problem(const psb_collider& o) {
    const int items = o.type == PSB_COLLIDER_MESH ? 12 : o.type == PSB_COLLIDER_HEIGHT ? 6 : 0;
    for (float x : o.v)
        if (!std::isfinite(x)) return "non-finite parameter";
    if (!std::isfinite(o.elast)) return "non-finite elast";
    switch (o.type) {
        case PSB_COLLIDER_PLANE:
        case PSB_COLLIDER_CYLINDER:
            return "";
        case PSB_COLLIDER_SPHERE:
            if (!o.container && o.elast > 0.f)
                return "a sphere with container = 0 and elast > 0 (the reference's restitution divides by zero)";
            return "";
        case PSB_COLLIDER_MESH:
        case PSB_COLLIDER_HEIGHT:
            if (o.count < 1 || o.count > PSB_MAX_COLLIDER_ITEMS || !o.data) return "count or data out of range";
            for (long long i = 0; i < (long long)o.count * items; ++i)
                if (!std::isfinite(o.data[i])) return "non-finite face or term";
            if (o.type == PSB_COLLIDER_HEIGHT)
                for (int i = 0; i < o.count; ++i) {
                    const float k = o.data[6 * i];
                    if (k != PSB_HEIGHT_LINEAR && k != PSB_HEIGHT_GAUSSIAN && k != PSB_HEIGHT_COSINE)
                        return "unknown height term kind";
                }
            return "";
        default:
            return "unknown type";
    }
}

void drop_colliders(psb_ctx* c) {
    cudaFree(c->d_coll);
    c->d_coll = nullptr;
    for (float* d : c->coll_data) cudaFree(d);
    c->coll_data.clear();
    c->P.coll = nullptr;
    c->P.n_coll = 0;
}

}  // namespace

int psb_emit(psb_ctx* c, int32_t k, const float* pos, const float* vel, const float* vel_half) {
    if (!c) return PSB_EINVAL;
    if (k <= 0 || !pos) return fail(c, PSB_EINVAL, "psb_emit: bad k or NULL pos");
    if (c->batch) return fail(c, PSB_EINVAL, "psb_emit: single-scene contexts only");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_emit before psb_upload");
    if ((int64_t)c->n + k > (int64_t)c->n_max)
        return fail(c, PSB_EINVAL, "psb_emit: " + std::to_string(k) + " particles, " +
                                       std::to_string(c->n_max - c->n) + " free of the context's capacity");
    enter(c);
    cudaStream_t st = c->stream;
    float* stage = (float*)c->stage;
    const int n0 = c->n;
    const float* vh = c->P.dem ? vel : vel_half;     // a DEM sphere's half-step velocity is its velocity
    struct { const float* src; float4* dst; } parts[3] = {
        {pos, c->pos[c->cs] + n0}, {vel, c->vel[c->cs] + n0}, {vh, c->vap[c->cs] + n0}};
    for (auto& p : parts) {
        if (p.src)
            PSB_TRY(cuda_check(c, cudaMemcpyAsync(stage, p.src, sizeof(float) * 3 * (size_t)k, cudaMemcpyHostToDevice,
                                                  st), "emit"));
        k_pack3<<<blocks(k), psb::kBlock, 0, st>>>(k, p.src ? stage : nullptr, p.dst);
    }
    psb::launch_append_ids(st, n0, k, c->ids[c->cr], c->rp[c->cr]);
    if (c->P.ext_force) cudaMemsetAsync(c->ext_force + n0, 0, sizeof(float4) * (size_t)k, st);
    c->n += k;
    c->built = false;
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "emit"));   // the host arrays are the caller's again
    return cuda_check(c, cudaGetLastError(), "emit");
}

int psb_add_emitter(psb_ctx* c, const psb_emitter* e) {
    if (!c) return PSB_EINVAL;
    if (!e) return fail(c, PSB_EINVAL, "psb_add_emitter: NULL emitter");
    if (c->batch) return fail(c, PSB_EINVAL, "psb_add_emitter: single-scene contexts only");
    if ((int)c->emitters.size() >= PSB_MAX_EMITTERS) return fail(c, PSB_EINVAL, "psb_add_emitter: too many emitters");
    if (e->duration < 0) return fail(c, PSB_EINVAL, "psb_add_emitter: negative duration");
    for (float x : e->v)
        if (!std::isfinite(x)) return fail(c, PSB_EINVAL, "psb_add_emitter: non-finite parameter");
    for (float x : e->velocity)
        if (!std::isfinite(x)) return fail(c, PSB_EINVAL, "psb_add_emitter: non-finite velocity");
    const bool lattice = e->type == PSB_EMITTER_BOX || e->type == PSB_EMITTER_SPHERE ||
                         e->type == PSB_EMITTER_CYLINDER;
    if (lattice && !(e->particle_radius > 0.f))
        return fail(c, PSB_EINVAL, "psb_add_emitter: particle_radius must be > 0");
    // One generation, stopped at the context's free capacity: an emission
    // that could never be appended is refused before it fills host memory.
    const int64_t free_slots = (int64_t)c->n_max - c->n;
    std::vector<float> xyz;
    const int g = psb::emit::generate(*e, 0, free_slots, xyz);
    if (g == PSB_EOVERFLOW_NBR)
        return fail(c, PSB_EINVAL, "psb_add_emitter: one emission exceeds the " + std::to_string(free_slots) +
                                       " free slots of the context's capacity");
    if (g == PSB_ENOMEM) return fail(c, PSB_ENOMEM, "psb_add_emitter: host memory for the emission");
    if (g != PSB_OK) return fail(c, PSB_EINVAL, "psb_add_emitter: bad type, count or faces");
    const int64_t per = (int64_t)(xyz.size() / 3);
    enter(c);
    EmitterRec r;
    r.e = *e;
    r.e.data = nullptr;
    r.per = per;
    const bool random = e->type == PSB_EMITTER_ELLIPSOID || e->type == PSB_EMITTER_MESH;
    int rc = PSB_OK;
    if (!random && per > 0) {
        rc = dalloc(c, &r.d_list, xyz.size());
        if (rc == PSB_OK)
            rc = cuda_check(c, cudaMemcpy(r.d_list, xyz.data(), sizeof(float) * xyz.size(), cudaMemcpyHostToDevice),
                            "emitter");
    } else if (e->type == PSB_EMITTER_MESH && e->n_faces > 0) {
        rc = dalloc(c, &r.d_faces, 9 * (size_t)e->n_faces);
        if (rc == PSB_OK)
            rc = cuda_check(c, cudaMemcpy(r.d_faces, e->data, sizeof(float) * 9 * (size_t)e->n_faces,
                                          cudaMemcpyHostToDevice), "emitter");
    }
    if (rc != PSB_OK) {
        cudaFree(r.d_list);
        cudaFree(r.d_faces);
        return rc;
    }
    c->emitters.push_back(r);
    return PSB_OK;
}

int psb_clear_emitters(psb_ctx* c) {
    if (!c) return PSB_EINVAL;
    enter(c);
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "emitters"));
    for (auto& e : c->emitters) { cudaFree(e.d_list); cudaFree(e.d_faces); }
    c->emitters.clear();
    return PSB_OK;
}

int psb_set_colliders(psb_ctx* c, const psb_collider* objs, int32_t n) {
    if (!c) return PSB_EINVAL;
    if (n < 0 || n > PSB_MAX_COLLIDERS || (n > 0 && !objs))
        return fail(c, PSB_EINVAL, "psb_set_colliders: bad argument");
    if (n > 0 && c->batch) return fail(c, PSB_EINVAL, "psb_set_colliders: single-scene contexts only");
    for (int i = 0; i < n; ++i) {
        const std::string why = collider_problem(objs[i]);
        if (!why.empty()) return fail(c, PSB_EINVAL, "psb_set_colliders: object " + std::to_string(i) + ": " + why);
    }
    enter(c);
    cudaStream_t st = c->stream;
    release_graphs(c);
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "colliders"));   // no step still reads the old list
    drop_colliders(c);
    if (n == 0) return PSB_OK;
    std::vector<psb::Collider> h((size_t)n);
    for (int i = 0; i < n; ++i) {
        const psb_collider& o = objs[i];
        psb::Collider& d = h[(size_t)i];
        d = psb::Collider{};
        d.type = o.type;
        d.flag = o.container ? 1 : 0;
        d.elast = o.elast;
        d.count = o.count;
        std::memcpy(d.v, o.v, sizeof d.v);
        if (o.type == PSB_COLLIDER_MESH || o.type == PSB_COLLIDER_HEIGHT) {
            const size_t m = (size_t)o.count * (o.type == PSB_COLLIDER_MESH ? 12 : 6);
            float* buf = nullptr;
            int rc = dalloc(c, &buf, m);
            if (rc == PSB_OK) {
                c->coll_data.push_back(buf);
                rc = cuda_check(c, cudaMemcpyAsync(buf, o.data, sizeof(float) * m, cudaMemcpyHostToDevice, st),
                                "colliders");
            }
            if (rc != PSB_OK) {
                cudaStreamSynchronize(st);
                drop_colliders(c);
                return rc;
            }
            if (o.type == PSB_COLLIDER_MESH) {
                d.fa = buf; d.fb = buf + 3; d.fc = buf + 6; d.fn = buf + 9;
                d.stride = 12;
            } else {
                d.terms = buf;
            }
        }
    }
    int rc = dalloc(c, &c->d_coll, (size_t)n);
    if (rc == PSB_OK)
        rc = cuda_check(c, cudaMemcpyAsync(c->d_coll, h.data(), sizeof(psb::Collider) * h.size(), cudaMemcpyHostToDevice,
                                           st), "colliders");
    if (rc == PSB_OK) rc = cuda_check(c, cudaStreamSynchronize(st), "colliders");
    if (rc != PSB_OK) {
        cudaStreamSynchronize(st);
        drop_colliders(c);
        return rc;
    }
    c->P.coll = c->d_coll;
    c->P.n_coll = n;
    return PSB_OK;
}

int psb_boundary_psi(psb_ctx* c, float* psi) {
    if (!c || !psi) return PSB_EINVAL;
    if (c->bnd_n == 0) return fail(c, PSB_ESTATE, "psb_boundary_psi: no boundary set");
    enter(c);
    cudaStream_t st = c->stream;
    std::vector<float> w((size_t)c->bnd_n);
    std::vector<int> ids((size_t)c->bnd_n);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(w.data(), c->bnd_w, sizeof(float) * w.size(), cudaMemcpyDeviceToHost, st), "psi"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(ids.data(), c->bnd_ids, sizeof(int) * ids.size(), cudaMemcpyDeviceToHost, st),
                       "psi"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "psi"));
    for (int t = 0; t < c->bnd_n; ++t) psi[ids[t]] = (float)(w[t] * c->sc.mass);
    return PSB_OK;
}

int psb_diagnostics(psb_ctx* c, psb_diag* out, int32_t n_out) {
    if (!c || !out) return PSB_EINVAL;
    if (n_out != 1 && n_out != c->nscenes) return fail(c, PSB_EINVAL, "psb_diagnostics: n_out is 1 or the scene count");
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_diagnostics before psb_upload");
    static_assert(sizeof(psb_diag) == sizeof(double) * psb::kDiagTerms, "psb_diag holds the diagnostic terms");
    enter(c);
    cudaStream_t st = c->stream;
    PSB_TRY(grow(c, &c->diag_rows, &c->diag_rows_cap, (long long)psb::diag_rows(c->n) * psb::kDiagTerms));
    PSB_TRY(grow(c, &c->diag_out, &c->diag_out_cap, (long long)n_out * psb::kDiagTerms));
    const float g[3] = {c->P.gx, c->P.gy, c->P.gz};
    for (int k = 0; k < n_out; ++k) {
        const int first = n_out == 1 ? 0 : (int)c->first[k];
        const int count = n_out == 1 ? c->n : (int)(c->first[k + 1] - c->first[k]);
        psb::launch_diagnostics(st, first, count, c->sc.mass, c->sc.rho0, g, c->pos[c->cs], c->vel[c->cs],
                                c->rp[c->cr], c->diag_rows, c->diag_out + (size_t)k * psb::kDiagTerms);
    }
    std::vector<double> h((size_t)n_out * psb::kDiagTerms);
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(h.data(), c->diag_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st),
                       "diagnostics"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "diagnostics"));
    for (int k = 0; k < n_out; ++k) {
        const double* r = &h[(size_t)k * psb::kDiagTerms];
        const double count = n_out == 1 ? (double)c->n : (double)(c->first[k + 1] - c->first[k]);
        out[k].mass = r[0];
        out[k].momentum[0] = r[1]; out[k].momentum[1] = r[2]; out[k].momentum[2] = r[3];
        out[k].kinetic = r[4];
        out[k].potential = r[5];
        out[k].density_err_mean = count > 0 ? r[6] / count : 0.0;
        out[k].density_err_max = r[7];
    }
    return cuda_check(c, cudaGetLastError(), "diagnostics");
}

int psb_iso_field(psb_ctx* c, const psb_iso_grid* g, double* iso) {
    if (!c) return PSB_EINVAL;
    psb::IsoParams Q;
    PSB_TRY(iso_on_device(c, g, 0.0, Q));
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (iso)
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(iso, c->iso, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream), "iso"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(c->stream), "iso"));
    return read_flags(c);
}

int psb_extract_surface(psb_ctx* c, const psb_iso_grid* g, double level, float* vertices, int64_t* n_vertices,
                        int32_t* triangles, int64_t* n_triangles) {
    if (!c || !n_vertices || !n_triangles) return PSB_EINVAL;
    psb::IsoParams Q;
    PSB_TRY(iso_on_device(c, g, level, Q));
    cudaStream_t st = c->stream;
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (!c->mc_table) {
        psb::mc_upload_table(st);
        c->mc_table = true;
    }
    // counts per cube (indexed by its lowest node) and per node edge, one
    // trailing zero each: their in-place exclusive scans end in the totals
    const long long cube_n = nn + 1, edge_n = 3 * nn + 1;
    PSB_TRY(grow(c, &c->mc_cube, &c->mc_cube_cap, cube_n));
    PSB_TRY(grow(c, &c->mc_edge, &c->mc_edge_cap, edge_n));
    PSB_TRY(grow(c, &c->mc_scratch, &c->mc_scratch_cap, psb::scan_scratch_words(edge_n)));
    timed(c, "mc_classify", [&] { psb::launch_mc_classify(st, Q, c->iso, c->mc_cube, c->mc_edge); });
    timed(c, "mc_scan", [&] {
        psb::scan_exclusive_u32(st, edge_n, c->mc_edge, c->mc_scratch);
        psb::scan_exclusive_u32(st, cube_n, c->mc_cube, c->mc_scratch);
    });
    uint32_t tot[2] = {0, 0};
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(&tot[0], c->mc_edge + 3 * nn, 4, cudaMemcpyDeviceToHost, st), "mc"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(&tot[1], c->mc_cube + nn, 4, cudaMemcpyDeviceToHost, st), "mc"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "mc"));
    const int64_t nv = tot[0], nt = tot[1];
    const bool fits = (!vertices || nv <= *n_vertices) && (!triangles || nt <= *n_triangles);
    *n_vertices = nv;
    *n_triangles = nt;
    if (!vertices && !triangles) return PSB_OK;
    if (!fits) return fail(c, PSB_EINVAL, "psb_extract_surface: output buffers too small (counts returned)");
    PSB_TRY(grow(c, &c->mc_vert, &c->mc_vert_cap, 3 * (nv > 0 ? nv : 1)));
    PSB_TRY(grow(c, &c->mc_tri, &c->mc_tri_cap, 3 * (nt > 0 ? nt : 1)));
    timed(c, "mc_emit", [&] { psb::launch_mc_emit(st, Q, c->iso, c->mc_edge, c->mc_cube, c->mc_vert, c->mc_tri); });
    if (vertices && nv)
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(vertices, c->mc_vert, sizeof(float) * 3 * nv, cudaMemcpyDeviceToHost, st), "mc"));
    if (triangles && nt)
        PSB_TRY(cuda_check(c, cudaMemcpyAsync(triangles, c->mc_tri, sizeof(int32_t) * 3 * nt, cudaMemcpyDeviceToHost, st), "mc"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "mc"));
    return cuda_check(c, cudaGetLastError(), "mc");
}

int psb_read_field(psb_ctx* c, int32_t field, void* dst, size_t bytes) {
    if (!c || !dst) return PSB_EINVAL;
    if (!c->uploaded) return fail(c, PSB_ESTATE, "psb_read_field before psb_upload");
    enter(c);
    cudaStream_t st = c->stream;
    const int n = c->n;
    const int* ids = c->ids[c->cr];
    size_t need = 0;
    const void* src = c->stage;
    switch (field) {
        case PSB_FIELD_POS: case PSB_FIELD_VEL: case PSB_FIELD_VEL_HALF: case PSB_FIELD_FORCE_NP: {
            const float4* s = field == PSB_FIELD_POS ? c->pos[c->cs] : field == PSB_FIELD_VEL ? c->vel[c->cs]
                            : field == PSB_FIELD_VEL_HALF ? c->vap[c->cs] : c->fnp;
            need = sizeof(float) * 3 * n;
            k_scatter3<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, s, (float*)c->stage);
            break;
        }
        case PSB_FIELD_DENSITY: case PSB_FIELD_PRESSURE:
            need = sizeof(float) * n;
            k_scatter_rp<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, c->rp[c->cr], field == PSB_FIELD_PRESSURE, (float*)c->stage);
            break;
        case PSB_FIELD_DENSITY_X:
            need = sizeof(float) * n;
            k_scatter_u32<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, (const uint32_t*)c->rho_x, (uint32_t*)c->stage);
            break;
        case PSB_FIELD_NBR_COUNT:
            need = sizeof(int) * n;
            k_scatter_u32<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, (const uint32_t*)c->nbr_count, (uint32_t*)c->stage);
            break;
        case PSB_FIELD_CELL_KEY:
            if (c->sorted < 0) return fail(c, PSB_ESTATE, "no sort yet");
            need = sizeof(uint32_t) * n;
            k_scatter_u32<<<blocks(n), psb::kBlock, 0, st>>>(n, ids, c->keys[c->sorted], (uint32_t*)c->stage);
            break;
        case PSB_FIELD_SORTED_ID:
            need = sizeof(int) * n;
            src = ids;
            break;
        case PSB_FIELD_SORTED_KEY:
            if (c->sorted < 0) return fail(c, PSB_ESTATE, "no sort yet");
            need = sizeof(uint32_t) * n;
            src = c->keys[c->sorted];
            break;
        default:
            return fail(c, PSB_EINVAL, "unknown field");
    }
    if (bytes < need) return fail(c, PSB_EINVAL, "destination too small");
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, st), "read_field"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "read_field"));
    return cuda_check(c, cudaGetLastError(), "read_field");
}

int psb_batch_layout(const psb_ctx* c, int32_t* n_scenes, int64_t* first) {
    if (!c) return PSB_EINVAL;
    if (n_scenes) *n_scenes = c->nscenes;
    if (first) std::copy(c->first.begin(), c->first.end(), first);
    return PSB_OK;
}

int psb_batch_stats(psb_ctx* c, int32_t* iters, int32_t* converged, double* err_final, int64_t* iters_total,
                    int64_t* unconverged_steps) {
    if (!c) return PSB_EINVAL;
    const int S = c->nscenes;
    if (!c->batch) {
        if (iters) iters[0] = c->stats.iters;
        if (converged) converged[0] = c->stats.converged;
        if (err_final) err_final[0] = c->stats.iters >= 0 && c->stats.iters <= PSB_MAX_ITERS ? c->stats.err[c->stats.iters] : 0.0;
        if (iters_total) iters_total[0] = c->stats.iters_total;
        if (unconverged_steps) unconverged_steps[0] = -1;
        return PSB_OK;
    }
    enter(c);
    cudaStream_t st = c->stream;
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_loop, c->d_loop, sizeof(int) * (2 + 4 * (size_t)S), cudaMemcpyDeviceToHost,
                                          st), "loop"));
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->h_err_sh, c->d_err_sh, sizeof(unsigned long long) * (PSB_MAX_ITERS + 1) * S,
                                          cudaMemcpyDeviceToHost, st), "err"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "sync"));
    for (int k = 0; k < S; ++k) {
        const int it = c->h_loop[2 + k];
        if (iters) iters[k] = it;
        if (converged) converged[k] = c->h_loop[2 + S + k];
        if (err_final) {
            // the last density pass: at index it if converged there, else it - 1
            const int last = c->h_loop[2 + S + k] ? it : it - 1;
            const unsigned long long e = last >= 0 && last <= PSB_MAX_ITERS ? c->h_err_sh[(size_t)last * S + k] : 0ull;
            err_final[k] = e ? psb::unorder_double(e) : 0.0;
        }
        if (iters_total) iters_total[k] = c->h_loop[2 + 2 * S + k];
        if (unconverged_steps) unconverged_steps[k] = c->h_loop[2 + 3 * S + k];
    }
    return PSB_OK;
}

int psb_set_graph(psb_ctx* c, int32_t on) {
    if (!c) return PSB_EINVAL;
    if (!c->batch && !(c->P.pci && !c->P.ref))
        return fail(c, PSB_EINVAL, "psb_set_graph: batches and config-profile PCISPH scenes only");
    enter(c);
    if (!on) release_graphs(c);
    c->graph_on = on != 0;
    return PSB_OK;
}

int psb_set_corrector(psb_ctx* c, int32_t mode) {
    if (!c) return PSB_EINVAL;
    if (!c->batch && !(c->P.pci && !c->P.ref))
        return fail(c, PSB_EINVAL, "psb_set_corrector: batches and config-profile PCISPH scenes only");
    if (mode != PSB_CORRECTOR_LAUNCHES && mode != PSB_CORRECTOR_PERSISTENT)
        return fail(c, PSB_EINVAL, "psb_set_corrector: unknown mode " + std::to_string(mode));
    enter(c);
    if (mode == PSB_CORRECTOR_PERSISTENT) {
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        if (!coop) return fail(c, PSB_ECUDA, "psb_set_corrector: the device has no cooperative launch");
    }
    if (mode != c->corrector) release_graphs(c);
    c->corrector = mode;
    return PSB_OK;
}

static bool block_ok(int b) { return b == 0 || b == 128 || b == 256 || b == 512; }

int psb_tune_set(psb_ctx* c, const psb_tune* t) {
    if (!c || !t) return PSB_EINVAL;
    if (t->bucket < 0 || t->bucket > 62 || !block_ok(t->nbr_block) || !block_ok(t->density_block) ||
        !block_ok(t->init_block) || !block_ok(t->pci_density_block) || !block_ok(t->force_block) ||
        !block_ok(t->xsph_block) || t->nbr_schedule < 0 || t->nbr_schedule > 2)
        return fail(c, PSB_EINVAL, "psb_tune_set: block sizes 0/128/256/512, schedule 0 or 1, bucket 0..62");
    enter(c);
    c->tune_table[t->bucket] = *t;
    release_graphs(c);
    apply_tune(c);
    return PSB_OK;
}

int psb_tune_get(psb_ctx* c, int32_t bucket, psb_tune* out) {
    if (!c || !out) return PSB_EINVAL;
    auto it = c->tune_table.find(bucket);
    if (it != c->tune_table.end()) { *out = it->second; return PSB_OK; }
    std::memset(out, 0, sizeof(*out));
    out->bucket = bucket;
    return PSB_OK;
}

int psb_autotune(psb_ctx* c, int32_t trials, psb_tune* out) {
    if (!c || trials < 1 || trials > 1000) return fail(c, PSB_EINVAL, "psb_autotune: trials in 1..1000");
    if (!c->uploaded || !c->built || c->sorted < 0 || c->stats.steps < 1)
        return fail(c, PSB_ESTATE, "psb_autotune: take a step first");
    enter(c);
    cudaStream_t st = c->stream;
    const int n = c->n;
    const int s = c->cs, r = c->cr;
    const bool pci = c->P.pci && !c->P.dem;
    const bool sph = !c->P.dem;
    const bool feats = pci && !c->P.ref && (c->sc.warm_start == PSB_WARM_LEARNED || c->collect_stride > 0);
    const int warm = (pci && (c->P.ref || c->sc.warm_start != PSB_WARM_ZERO)) ? 1 : 0;
    // the pressure-force pass overwrites the carried pressures, the density
    // pass the densities: keep them
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->stage, c->rp[r], sizeof(float2) * n, cudaMemcpyDeviceToDevice, st), "tune"));
    if (c->batch) cudaMemsetAsync(c->d_active, 1, c->nscenes, st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // In a step every kernel finds the data its predecessor left in L2, not
    // its own; back-to-back repeats would favour configurations that reuse a
    // warm L2. Each timed launch follows a write of 256 MB (twice L2).
    const size_t flush_bytes = (size_t)256 << 20;
    void* flush = nullptr;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) { cudaGetLastError(); flush = nullptr; }
    auto time_it = [&](auto launch) {
        launch();
        double total = 0.0;
        for (int i = 0; i < trials; ++i) {
            if (flush) cudaMemsetAsync(flush, i & 0xff, flush_bytes, st);
            cudaEventRecord(e0, st);
            launch();
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        return total / trials;
    };
    const int blocks[3] = {128, 256, 512};
    psb_tune best{};
    best.bucket = size_bucket(n);
    Params P = c->P;
    P.n = n;
    // one kernel at a time: every other kernel at its default
    auto tune_one = [&](int which, auto launch) {
        double best_ms = 1e300;
        int best_b = 256, best_sched = 0;
        const int nsched = which == 0 ? (can_fuse_density(c, P) ? 3 : 2) : 1;
        for (int sched = 0; sched < nsched; ++sched)
            for (int b : blocks) {
                Params Q = P;
                Q.tune = psb::Tune{};
                switch (which) {
                    case 0: Q.tune.nbr_block = b; Q.tune.nbr_schedule = sched; break;
                    case 1: Q.tune.density_block = b; break;
                    case 2: Q.tune.init_block = b; break;
                    case 3: Q.tune.pci_density_block = b; break;
                    case 4: Q.tune.force_block = b; break;
                    default: Q.tune.xsph_block = b; break;
                }
                const double ms = time_it([&] { launch(Q); });
                if (b == 256 && sched == 0) best.ms_default[which] = ms;
                if (ms < best_ms) { best_ms = ms; best_b = b; best_sched = sched; }
            }
        best.ms[which] = best_ms;
        switch (which) {
            case 0: best.nbr_block = best_b; best.nbr_schedule = best_sched; break;
            case 1: best.density_block = best_b; break;
            case 2: best.init_block = best_b; break;
            case 3: best.pci_density_block = best_b; break;
            case 4: best.force_block = best_b; break;
            default: best.xsph_block = best_b; break;
        }
    };
    // The neighbour build. Where the density pass at x can fold into it,
    // every schedule is timed with that pass: schedules 0 and 1 followed by
    // the separate pass (at its default block), schedule 2 the fused kernel,
    // so that all three do the same work.
    tune_one(0, [&](const Params& Q) {
        if (fused_density(c, Q)) {
            psb::launch_build_density(st, Q, c->pos[s], c->vel[s], c->keys[c->sorted], c->cell_start, c->cell_end,
                                      c->nbr_count, c->nbr_list, c->flags, c->rp[r], c->rho_x, 0, c->p_scale,
                                      feats ? c->feats : nullptr, psb::mlp_inputs(c->mlp_arch));
            return;
        }
        psb::launch_build_nbr(st, Q, c->pos[s], c->keys[c->sorted], c->cell_start, c->cell_end, c->nbr_count,
                              c->nbr_list, c->flags);
        if (can_fuse_density(c, Q)) {
            Params D = Q;
            D.tune = psb::Tune{};
            psb::launch_density_x(st, D, c->pos[s], c->vel[s], c->nbr_count, c->nbr_list, c->rp[r], c->rho_x, 0,
                                  c->p_scale, feats ? c->feats : nullptr, psb::mlp_inputs(c->mlp_arch));
        }
    });
    if (sph)
        tune_one(1, [&](const Params& Q) {
            psb::launch_density_x(st, Q, c->pos[s], c->vel[s], c->nbr_count, c->nbr_list, c->rp[r], c->rho_x, 0,
                                  c->p_scale, feats ? c->feats : nullptr, psb::mlp_inputs(c->mlp_arch));
        });
    if (pci) {
        tune_one(2, [&](const Params& Q) {
            psb::launch_pci_init(st, Q, c->pos[s], c->vel[s], c->vap[s], c->rp[r], c->nbr_count, c->nbr_list, warm,
                                 c->fnp, c->xs[0], c->vs);
        });
        tune_one(3, [&](const Params& Q) {
            psb::launch_pci_density(st, Q, c->xs[0], c->rp[r], c->nbr_count, c->nbr_list, c->rpc, &c->err_hist[0]);
        });
        tune_one(4, [&](const Params& Q) {
            psb::launch_pci_force_predict(st, Q, c->pos[s], c->vap[s], c->fnp, c->xs[0], c->rpc, c->nbr_count,
                                          c->nbr_list, c->xs[1], c->vs, c->rp[r]);
        });
        tune_one(5, [&](const Params& Q) {
            psb::launch_xsph(st, Q, c->xs[0], c->vs, c->nbr_count, c->nbr_list, c->xs[1]);
        });
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (flush) { cudaStreamSynchronize(st); cudaFree(flush); }
    PSB_TRY(cuda_check(c, cudaMemcpyAsync(c->rp[r], c->stage, sizeof(float2) * n, cudaMemcpyDeviceToDevice, st), "tune"));
    PSB_TRY(cuda_check(c, cudaStreamSynchronize(st), "tune"));
    PSB_TRY(cuda_check(c, cudaGetLastError(), "tune"));
    // kernels a scene does not run keep the default
    if (!sph) best.density_block = 0;
    if (!pci) best.init_block = best.pci_density_block = best.force_block = best.xsph_block = 0;
    c->tune_table[best.bucket] = best;
    release_graphs(c);
    apply_tune(c);
    if (out) *out = best;
    return PSB_OK;
}

int psb_context_info(const psb_ctx* c, psb_scene* scene, int32_t* n, int64_t* steps) {
    if (!c) return PSB_EINVAL;
    if (scene) *scene = c->sc;
    if (n) *n = c->uploaded ? c->n : 0;
    if (steps) *steps = c->stats.steps;
    return PSB_OK;
}

int psb_set_step_count(psb_ctx* c, int64_t steps) {
    if (!c || steps < 0) return PSB_EINVAL;
    c->stats.steps = steps;
    return PSB_OK;
}

int psb_get_stats(psb_ctx* c, psb_step_stats* out) {
    if (!c || !out) return PSB_EINVAL;
    *out = c->stats;
    return PSB_OK;
}

int psb_profile_enable(psb_ctx* c, int32_t on) {
    if (!c) return PSB_EINVAL;
    c->prof.resolve(c->stream);
    c->prof.on = on != 0;
    return PSB_OK;
}

int psb_profile_read(psb_ctx* c, int32_t index, char* name, size_t name_len, int64_t* launches, double* ms) {
    if (!c) return PSB_EINVAL;
    c->prof.resolve(c->stream);
    if (index < 0 || index >= (int)c->prof.names.size()) return PSB_EINVAL;
    if (name && name_len) {
        std::strncpy(name, c->prof.names[index].c_str(), name_len - 1);
        name[name_len - 1] = 0;
    }
    if (launches) *launches = c->prof.launches[index];
    if (ms) *ms = c->prof.ms[index];
    return PSB_OK;
}

int psb_profile_reset(psb_ctx* c) {
    if (!c) return PSB_EINVAL;
    c->prof.resolve(c->stream);
    std::fill(c->prof.launches.begin(), c->prof.launches.end(), 0);
    std::fill(c->prof.ms.begin(), c->prof.ms.end(), 0.0);
    return PSB_OK;
}

}  // extern "C"
