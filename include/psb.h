/*
 * psb.h -- C ABI of the B200 particle-simulation hot path (libpsb.so).
 *
 * Plain C: opaque context, plain pointers and sizes, int status returns,
 * caller-owned host buffers, library-owned device buffers, one CUDA stream
 * per context. Everything is asynchronous on that stream except the calls
 * that return host data (psb_download*, psb_read_field, psb_get_stats) and
 * psb_step, which reads the corrector loop's convergence word each
 * iteration.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the edarles/PSB_Project tree). The reference's system classes
 * (PCI_SPHSystem, SPHSystem) keep their class API; their update() bodies
 * call these functions instead of the reference launchers. The Python
 * package (psb_project_b200/runtime.py) binds the same functions with ctypes.
 */
#ifndef PSB_H
#define PSB_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSB_ABI_VERSION 2

/* Status codes. The reference's launchers return void and never check
 * (src/common.cu:63-66); every call here returns one of these. */
enum {
    PSB_OK = 0,
    PSB_EINVAL = 1,          /* bad argument or scene */
    PSB_ENOMEM = 2,          /* device or host allocation failed */
    PSB_EOVERFLOW_NBR = 3,   /* a particle had more neighbours than scene.nbr_cap */
    PSB_ENOCONV = 4,         /* corrector loop hit max_iters above eta (state is still advanced) */
    PSB_ECUDA = 5,           /* CUDA runtime error */
    PSB_ESTATE = 6           /* call out of order (e.g. step before upload) */
};

/* Physics profiles. REF reproduces the reference's formulas (linear EOS,
 * surface tension, fixed 3 corrector passes, projection walls, hard-coded
 * -9.81 y gravity in PCISPH). CONFIG is the scene text's method (Tait EOS,
 * penalty walls, eta loop with min/max iterations, no surface tension). */
enum { PSB_PROFILE_REF = 0, PSB_PROFILE_CONFIG = 1 };
/* PSB_DEM: the reference's discrete-element system (CudaSystem::update,
 * CudaSystem.cpp:207-224): spheres with pairwise spring-dashpot contacts
 * over the same grid and neighbour lists, gravity, explicit Euler, walls. */
enum { PSB_WCSPH = 0, PSB_PCISPH = 1, PSB_DEM = 2 };
/* Initial pressure of each PCISPH step (CONFIG profile). */
enum { PSB_WARM_ZERO = 0, PSB_WARM_PREVIOUS = 1, PSB_WARM_LEARNED = 2 };

/* Scene: the uniform per-particle parameters the reference keeps in
 * per-particle arrays (SimulationData_SPHSystem.cpp:5-16), the grid of
 * UniformGrid (UniformGrid.cuh:16-33: float Min, float sizeCell, cell
 * counts) and the container box of BoxCollision. */
typedef struct psb_scene {
    int32_t n_max;              /* particle capacity */
    float box_min[3], box_max[3];
    float grid_min[3];          /* grid corner */
    float cell;                 /* cell edge, >= h */
    int32_t dims[3];            /* cells per axis */
    double h;                   /* smoothing radius = interaction radius */
    double mass, rho0, k, mu, sigma, l;
    float particle_radius;      /* wall offset */
    float dt;
    float gravity[3];           /* acceleration, CONFIG profile and WCSPH */
    int32_t profile, method;
    int32_t min_iters, max_iters;
    double eta;                 /* max (rho*-rho0)/rho0 accepted by the corrector loop */
    double wall_k, wall_c;      /* penalty walls, 1/s^2 and 1/s */
    int32_t nbr_cap;            /* neighbour slots per particle (0: 128) */
    int32_t warm_start;         /* PSB_WARM_* */
    double spacing;             /* rest lattice spacing of the CONFIG-profile PCISPH prototype
                                   (0: (mass/rho0)^(1/3)) */
    double skin;                /* CONFIG profile: neighbour lists hold every pair within (1 + skin) h,
                                   so pairs that close in during the step's predictions are in them
                                   (kernels still cut off at h); cell must be >= (1 + skin) h.
                                   REF profile: must be 0 (the reference's test is r <= h). */
    double xsph;                /* CONFIG-profile PCISPH: XSPH velocity smoothing after the corrector,
                                   v_i += xsph sum_j (m/rho0) W_ij (v_j - v_i) at the committed
                                   positions (Monaghan 1989); 0 = off, at most 1. REF profile: 0. */
    /* PSB_DEM contact law. REF profile: collideParticle (CudaParticle_Kernel.cu:
     * 10-36) as it executes: -dem_spring (R - d) n for d < 2R, R = h_A + h_B
     * with h the interaction radius, which interactionSystem passes as the
     * sphere radius (CudaSystem.cpp:244). Its damping, shear and attraction
     * terms are `force += ...` through a double3 operator+= that does not
     * assign (double3.h:115-117), so they have no effect there either.
     * CONFIG profile: linear spring-dashpot on overlaps of particle_radius
     * spheres, dem_spring = k_n (N/m), dem_damping = normal dashpot c_n
     * (N s/m); shear and attraction unused. mass is the sphere mass. */
    double dem_spring, dem_damping, dem_shear, dem_attraction;
} psb_scene;

#define PSB_MAX_ITERS 64
typedef struct psb_step_stats {
    int32_t iters;              /* pressure corrections in the last step */
    int32_t converged;
    int32_t nbr_max;            /* largest neighbour count (self included) */
    int32_t clamped;            /* particles whose cell was clamped into the grid */
    int64_t nbr_total;
    double err[PSB_MAX_ITERS + 1];   /* max (rho*-rho0)/rho0 of each density pass, FP64 */
    int64_t steps;              /* steps taken by this context */
    int64_t iters_total;        /* corrections summed over all steps */
} psb_step_stats;

typedef struct psb_ctx psb_ctx;

/* Fields psb_read_field can copy out, in particle-id order. */
enum {
    PSB_FIELD_POS = 0,          /* float x3 */
    PSB_FIELD_VEL = 1,          /* float x3, interpolated velocity (m_dVel[1]) */
    PSB_FIELD_VEL_HALF = 2,     /* float x3, leap-frog velocity (m_dVelInterAp) */
    PSB_FIELD_DENSITY = 3,      /* float: last density pass */
    PSB_FIELD_PRESSURE = 4,     /* float */
    PSB_FIELD_DENSITY_X = 5,    /* float: density at the step's start positions */
    PSB_FIELD_FORCE_NP = 6,     /* float x3: non-pressure force density */
    PSB_FIELD_NBR_COUNT = 7,    /* int32: neighbours incl. self */
    PSB_FIELD_CELL_KEY = 8,     /* uint32: cell index */
    PSB_FIELD_SORTED_ID = 9,    /* int32: particle id at each sorted slot (slot order, not id order) */
    PSB_FIELD_SORTED_KEY = 10   /* uint32: cell index at each sorted slot (slot order) */
};

/* Replaces SPHSystem::init/PCI_SPHSystem's constructor allocations
 * (SphSystem.cpp:57-113, PciSphSystem.cpp:7-24) and createGrid
 * (UniformGrid.cu:17-49): sizes every buffer from the scene, no fixed caps. */
int psb_create(const psb_scene* scene, psb_ctx** out);
int psb_destroy(psb_ctx* ctx);

/* Launch all work on `stream` (a cudaStream_t); NULL = the legacy stream.
 * Work later queued on the new stream waits for what the context had queued
 * on the previous one. */
int psb_set_stream(psb_ctx* ctx, void* stream);

/* Replaces the particle upload of PCI_SPHSystem::_initialize
 * (PciSphSystem.cpp:68-138): host arrays, particle-id order, xyz stride 3.
 * vel/vel_half may be NULL (zero). pressure may be NULL (zero).
 * Asynchronous: the positions are copied on the context's stream, the other
 * arrays on a copy stream of the context's own, and the next psb_step runs
 * its grid, sort and neighbour build while they are still in flight (it
 * waits for them before it first reads them). Every other call waits for
 * them first. From pinned host memory the copies overlap that work and run
 * after the call returns: keep the arrays unchanged until a call that waits
 * for the device (psb_step, psb_download, psb_read_field) has returned. */
int psb_upload(psb_ctx* ctx, int32_t n, const float* pos, const float* vel, const float* vel_half,
               const float* pressure);

/* Same, from the reference's AoS double3 layout (m_hPos[1], m_hVel[1],
 * m_hVelInterAp), converted once at this boundary. on_device != 0: the
 * pointers are device memory (the reference's m_dPos[1] etc.). */
int psb_upload_aos_f64(psb_ctx* ctx, int32_t n, const double* pos, const double* vel, const double* vel_half,
                       int32_t on_device);

/* Replaces the per-step device-to-host copies of interpolateVelocities
 * (SphSystem.cpp:337-345). Any pointer may be NULL. Blocks until done; the
 * copy of each array overlaps the reordering of the next. */
int psb_download(psb_ctx* ctx, float* pos, float* vel, float* vel_half, float* density, float* pressure);
int psb_download_aos_f64(psb_ctx* ctx, double* pos, double* vel, double* vel_half, int32_t on_device);

/* Replaces PCI_SPHSystem::update (PciSphSystem.cpp:163-204) and
 * SPHSystem::update (SphSystem.cpp:273-297) minus emission: grid, sort,
 * neighbours, the SPH/PCISPH step, walls, velocity interpolation. */
int psb_step(psb_ctx* ctx, int32_t nsteps);

/* Initial pressure for a CONFIG-profile PCISPH scene: `iters` corrector
 * passes at the current state with eta = 0, keeping positions and
 * velocities and only the pressure; with a warm start the following steps
 * begin from it. The reference has no counterpart (it restarts every step
 * from p = 0, PciSphSystem_Kernel.cu:131). stats.err[k] is pass k's error. */
int psb_presolve(psb_ctx* ctx, int32_t iters);

/* Replaces reinitCells + storeParticles + searchNeighbooring
 * (UniformGrid.cu:64-99, UniformGridKernel.cu:30-95): cell keys, stable
 * sort by (cell, id), cell ranges and neighbour lists at the current
 * positions, then the density there (compute_Density_PCI,
 * PciSphSystem_Kernel.cu:70-85). */
int psb_build_neighbors(psb_ctx* ctx);

/* Node grid of the iso field and the marching cubes: dims[a] nodes along
 * axis a at origin[a] + i spacing[a], x fastest. Replaces
 * createGrid_MarchingCube_CUDA (MarchingCube.cu:12-27), whose nodes sit at
 * centre - L/2 + sizeCell/2 + i sizeCell. */
typedef struct psb_iso_grid {
    double origin[3];
    double spacing[3];
    int32_t dims[3];
    double scale;               /* REF profile: evaluateIso's scale -- influence radius h/scale over
                                   floor(1/scale) rings of particle-grid cells (SurfaceSPH::extract
                                   uses 0.65, SurfaceSPH.cpp:31); finite and >= 1/16, and
                                   origin/spacing finite, or PSB_EINVAL */
} psb_iso_grid;

/* The iso field at every node of `grid`, at the current positions (the
 * particle grid is rebuilt first). REF profile: evaluateIso_Kernel
 * (UniformGridKernel.cu:98-138), sum over particles within r = h/scale of
 * (r^2 - d^2)^3 / r^6. CONFIG profile: the density-based colour field
 * sum_j (m/rho_j) W_poly6(|x - x_j|, h). iso: host buffer of
 * dims[0] dims[1] dims[2] doubles (NULL: leave it on the device). SPH scenes
 * only. */
int psb_iso_field(psb_ctx* ctx, const psb_iso_grid* grid, double* iso);

/* Marching cubes at `level` over the iso field of `grid`; replaces
 * polygonize_MarchingCube_CUDA (MarchingCube.cu:31-46) and the host vertex
 * weld of SurfaceSPH::extract (SurfaceSPH.cpp:120-186). Corner and edge
 * numbering, the case bit (iso <= level) and the vertex interpolation are
 * the reference's; the triangle table is generated from the cube's faces,
 * and every grid edge owns one vertex, so the mesh comes out welded.
 * On entry *n_vertices and *n_triangles are the capacities of `vertices`
 * (float x3 each) and `triangles` (int32 x3 vertex indices, normals toward
 * iso <= level); on return they are the counts. With both buffers NULL only
 * the counts are returned; a buffer too small gives PSB_EINVAL with the
 * counts set. */
int psb_extract_surface(psb_ctx* ctx, const psb_iso_grid* grid, double level, float* vertices,
                        int64_t* n_vertices, int32_t* triangles, int64_t* n_triangles);

/* Copies one field out (see PSB_FIELD_*); `bytes` is the destination size. */
int psb_read_field(psb_ctx* ctx, int32_t field, void* dst, size_t bytes);

int psb_get_stats(psb_ctx* ctx, psb_step_stats* out);

/* Per-kernel CUDA-event timing: enable, then read accumulated
 * (launches, milliseconds) per kernel name. */
int psb_profile_enable(psb_ctx* ctx, int32_t on);
int psb_profile_read(psb_ctx* ctx, int32_t index, char* name, size_t name_len, int64_t* launches, double* ms);
int psb_profile_reset(psb_ctx* ctx);

/* Host-side scene generator: lattice block with ids x-fastest, positions
 * origin + (i+0.5)*spacing + jitter, jitter uniform in [-J, J) from
 * SplitMix64(seed ^ (3*(id+id0)+axis)), rounded once to float. xyz stride 3.
 * Stands in for the reference's EmitterBox (EmitterBox.cpp:29-47). */
int psb_lattice(const int32_t nxyz[3], double spacing, const double origin[3], double jitter, uint64_t seed,
                int32_t id0, float* pos);

/* Allocation-free sort. No counterpart in the reference: its launchers take
 * buffers the caller allocated up front and keep no scratch.
 *
 * Sorts n (key, value) pairs of device memory stably by key (the same LSD
 * radix sort psb_step uses for (cell, id) ordering), reading keys_in/vals_in
 * and writing keys_out/vals_out; key_bits (1..32) bounds the keys. For
 * callers that cannot allocate device memory -- hosts that give the whole
 * GPU to their own memory pool and forbid libraries from allocating, and
 * per-frame loops that must not stall on cudaMalloc/cudaFree, which can
 * synchronise the device -- it calls no allocator: its scratch is a static
 * device array inside libpsb, held by every GPU that loads the library
 * (about 2.1 MB) until the process exits.
 * Limit: n <= PSB_NOALLOC_MAX_N; larger n returns PSB_EINVAL (with a message
 * on stderr). Every call looks up the array's address on the current device
 * (a host-side lookup), so the entry point stays valid after the host resets
 * the device. Sorting in place (keys_out == keys_in and/or vals_out ==
 * vals_in) is supported; any other overlap of the four ranges returns
 * PSB_EINVAL. A CUDA error already pending when the call starts is left in
 * place and the call returns PSB_ECUDA without running. All calls share the
 * one array: calls that overlap on the GPU (other streams or threads on the
 * same device) race and corrupt each other's results. */
#define PSB_NOALLOC_MAX_N 262144
int psb_sort_cells_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                           uint32_t* vals_out, int32_t n, int32_t key_bits, void* stream);

/* Learned warm start (CONFIG-profile PCISPH, warm_start = PSB_WARM_LEARNED):
 * a per-particle MLP with BF16 weights and activations and FP32
 * accumulation predicts each step's initial pressure; the corrector still
 * iterates to the same eta. No counterpart in the reference, which starts
 * every step from p = 0 (PciSphSystem_Kernel.cu:131). Two networks:
 *   PSB_MLP_SILU6 (the default): 6 -> 64 -> 64 -> 1, SiLU, 4,673 parameters;
 *   PSB_MLP_RELU7: 7 -> 64 -> 64 -> 1, ReLU, 4,737 parameters.
 * Parameters (FP32 master copy), in order: W1[64][n_in], b1[64],
 * W2[64][64], b2[64], W3[64], b3. Inputs, in order: neighbour count,
 * advected density, velocity divergence, previous pressure, wall distance,
 * density-gradient magnitude (the six of PSB_MLP_SILU6), and for
 * PSB_MLP_RELU7 the previous pressure smoothed with the poly6 weights over
 * the neighbours (scaled as in psb_project_b200/csrc/sph.cu, k_density_x).
 * Feature rows are PSB_MLP_FEATURE_STRIDE floats; the network reads the
 * first n_in. */
#define PSB_MLP_SILU6 0
#define PSB_MLP_RELU7 1
#define PSB_MLP_PARAMS 4737          /* the larger network's count: a buffer of this size fits either */
#define PSB_MLP_PARAMS_SILU6 4673
#define PSB_MLP_FEATURE_STRIDE 8
/* Selects the network; clears the weights and the optimiser state (set new
 * weights before stepping with the learned start or training). */
int psb_mlp_set_arch(psb_ctx* ctx, int32_t arch);
/* The context's network, its input count and its parameter count (any
 * pointer may be NULL). */
int psb_mlp_info(const psb_ctx* ctx, int32_t* arch, int32_t* n_inputs, int32_t* n_params);
/* The first half of a step, without stepping: rebuilds the grid and lists
 * at the current state and returns, in particle-id order, the warm start's
 * inputs (features: n rows of PSB_MLP_FEATURE_STRIDE floats, the first
 * n_in set) and the initial pressure the next psb_step starts its
 * corrector from (pressure: n floats; the network's prediction with
 * PSB_WARM_LEARNED, the carried pressure with PSB_WARM_PREVIOUS, 0 with
 * PSB_WARM_ZERO). Either pointer may be NULL. The state is unchanged, so a
 * psb_step that follows starts from exactly these values. Single
 * config-profile PCISPH contexts only. */
int psb_warm_start(psb_ctx* ctx, float* features, float* pressure);
/* The weights of the context's network (psb_mlp_info's n_params floats). */
int psb_mlp_set_weights(psb_ctx* ctx, const float* w);
int psb_mlp_get_weights(psb_ctx* ctx, float* w);
/* Record (features, converged pressure / p_scale) of every stride-th particle
 * after each converged step into a device ring of `capacity` rows; stride 0
 * stops recording. */
int psb_mlp_collect(psb_ctx* ctx, int32_t stride, int64_t capacity);
/* Rows recorded so far (capped at the capacity); X (rows x 8) and T (rows)
 * may be NULL, else receive the rows. */
int psb_mlp_dataset(psb_ctx* ctx, int64_t* rows, float* X, float* T);
/* `iters` Adam steps (lr, beta 0.9/0.999) on MSE over minibatches of `batch`
 * rows drawn from the recorded data; *loss = last minibatch loss. */
int psb_mlp_train(psb_ctx* ctx, int32_t iters, int32_t batch, float lr, uint64_t seed, float* loss);
/* Forward pass and loss gradient on host rows (X: n x 8, first 7 used; T: n
 * targets), for checking the GPU's arithmetic. */
int psb_mlp_forward(psb_ctx* ctx, const float* X, int32_t n, float* y);
int psb_mlp_loss_grad(psb_ctx* ctx, const float* X, const float* T, int32_t n, float* loss, float* grad);

/* Batched scenes: n_scenes independent scenes stepped together in one
 * context, each sweep one kernel launch over every scene's particles. No
 * counterpart in the reference, which steps one system per update
 * (PciSphSystem.cpp:163-204).
 * Every scene is CONFIG-profile PCISPH, and all share h, mass, rho0, dt, mu,
 * k, gravity, spacing, skin, xsph, cell, wall_k, wall_c, particle_radius,
 * eta, min_iters, max_iters, nbr_cap and warm_start; their boxes, grids
 * (grid_min, dims) and particle counts (n_max) differ. The particles are
 * concatenated in scene order: ids [0, n_max of scene 0) are scene 0, the
 * next n_max of scene 1 are scene 1, and so on; psb_upload takes exactly the
 * total and psb_download returns it in the same order.
 * Each scene gets its own grid and key range, its own convergence test and
 * corrector iteration count, and its own walls: its results are those it has
 * when stepped alone, bit for bit. The corrector loop runs on the device (a
 * one-block kernel tests each scene after every density pass and retires
 * the converged ones), so a step never waits on the host.
 * psb_step_stats of a batch: iters = the most corrections any scene took,
 * converged = all scenes converged, err = the max over scenes per pass. */
int psb_create_batch(const psb_scene* scenes, int32_t n_scenes, psb_ctx** out);
/* Scenes in the context (1 for psb_create) and the first particle id of each
 * (first: n_scenes + 1 entries, the last one the total; may be NULL). */
int psb_batch_layout(const psb_ctx* ctx, int32_t* n_scenes, int64_t* first);
/* Per-scene results (arrays of n_scenes, any may be NULL): the last step's
 * corrections, converged flag and final density-pass max error; and, since
 * the last upload, corrections summed over steps and the count of steps
 * that ended at max_iters unconverged (-1 for a single-scene context). */
int psb_batch_stats(psb_ctx* ctx, int32_t* iters, int32_t* converged, double* err_final, int64_t* iters_total,
                    int64_t* unconverged_steps);
/* CUDA-graph stepping (batches and config-profile PCISPH scenes; other
 * scenes return PSB_EINVAL): on, each step after the first since an upload
 * is one cudaGraphLaunch of the whole step, grid rebuild, warm start, the
 * corrector as a conditional while node (cudaGraphCondTypeWhile) and the
 * commit. Graphs are captured on first use, one per state buffer parity,
 * recaptured after emissions change the particle count, and released by
 * psb_set_graph(ctx, 0) and psb_destroy. Steps that record training data,
 * emit particles or run with profiling on are launched kernel by kernel,
 * the corrector deciding on the device with one 4-byte read per pass; both
 * ways launch the same kernels in the same order. */
int psb_set_graph(psb_ctx* ctx, int32_t on);

/* The corrector loop of batches and config-profile PCISPH scenes (others
 * return PSB_EINVAL). PSB_CORRECTOR_LAUNCHES (the default): three kernels
 * per correction, {density pass, decision, pressure-force pass}, repeated by
 * the graph's while node or by the host. PSB_CORRECTOR_PERSISTENT: the whole
 * loop in one cooperative launch of one resident wave of blocks, grid-wide
 * barriers in place of the kernel boundaries. Both run the same passes in
 * the same order on the same data: the results are bit-identical. */
#define PSB_CORRECTOR_LAUNCHES 0
#define PSB_CORRECTOR_PERSISTENT 1
int psb_set_corrector(psb_ctx* ctx, int32_t mode);

/* Autotuner: the launch configuration of the neighbour build and the five
 * gather sweeps (density at x, PCISPH set-up, density/pressure pass,
 * pressure-force pass, XSPH), kept per size bucket, bucket = floor(log2 n)
 * of the particle count (a batch's total). Candidates: block sizes 128, 256
 * and 512, and for the neighbour build three cell schedules -- 0, each
 * thread walks its own 27 cells; 1, the lanes of a warp that share a grid
 * row walk it together, staging 32 candidates at a time in shared memory;
 * 2, schedule 0 with the density pass at x (and the network's inputs) folded
 * into the same walk (single config-profile PCISPH scenes; elsewhere it runs
 * as 0). Where the fold is possible, schedules 0 and 1 are timed together
 * with the separate density pass. Every candidate computes the same result
 * bit for bit; only the time differs.
 * No counterpart in the reference, whose launches are sized by
 * computeGridSize with 256 threads (common.cu:102-107). */
typedef struct psb_tune {
    int32_t bucket;
    int32_t nbr_block, nbr_schedule;
    int32_t density_block, init_block, pci_density_block, force_block, xsph_block;
    /* mean launch times (ms) of the choice and of the default (256 threads,
     * schedule 0): neighbour build, density at x, set-up, density/pressure,
     * pressure force, XSPH (0 where the scene has no such kernel) */
    double ms[6];
    double ms_default[6];
} psb_tune;
/* Times every candidate `trials` times (CUDA events, after one untimed
 * launch, each timed launch after a 256 MB write that evicts L2, as in a
 * step no kernel finds its own data in L2) on the context's current
 * particles -- after at least one step --
 * and stores the fastest of each kernel for the current bucket; later steps
 * at that bucket use it. The state (positions, velocities, densities,
 * pressures) is left as it was; scratch buffers are recomputed next step.
 * Captured step graphs are released (they are captured again). */
int psb_autotune(psb_ctx* ctx, int32_t trials, psb_tune* out);
/* Installs a table entry (t->bucket; block sizes 0/128/256/512, 0 = 256;
 * schedule 0 or 1), e.g. one saved from an earlier run. */
int psb_tune_set(psb_ctx* ctx, const psb_tune* t);
/* The entry for `bucket` (block sizes 0 when the bucket has none). */
int psb_tune_get(psb_ctx* ctx, int32_t bucket, psb_tune* out);

/* Static boundary particles (CONFIG profile, single-scene SPH contexts),
 * after Akinci et al. 2012: a solid obstacle sampled by n_bnd particles
 * (pos: n_bnd x 3 floats, inside the grid). Each gets psi_b = rho0 /
 * sum_k W(x_b - x_k) over the boundary particles; a fluid particle gains
 * psi_b W in its density and psi_b p_i/rho0^2 gradW in its pressure force
 * (its own pressure mirrored onto the solid); free slip. Sample a solid at
 * least h thick (e.g. a shell of two lattice spacings). Replaces any earlier
 * set; n_bnd = 0 removes it. No counterpart in the reference, whose
 * obstacles are analytic collision objects (src/Kernel/Collision). */
int psb_set_boundary(psb_ctx* ctx, int32_t n_bnd, const float* pos);
/* psi_b (kg) of the current boundary set, in the order it was given. */
int psb_boundary_psi(psb_ctx* ctx, float* psi);
/* The force (N, n_bnd x 3, in the order given) the fluid exerts on each
 * boundary particle after the last step: minus the mirrored-pressure forces
 * the particle exerts on the fluid particles within h, from their committed
 * positions and pressures. With DEM spheres as the boundary particles this
 * is the fluid's side of a two-way coupling (C1). No counterpart in the
 * reference, which has no fluid-solid coupling. */
int psb_boundary_forces(psb_ctx* ctx, float* force);
/* Makes the current boundary set move with the pressure corrector (config
 * PCISPH, single scene): the two-way fluid-solid coupling solved inside the
 * step instead of staggered between steps. vel and force (n_bnd x 3, in the
 * order the set was given) are each particle's velocity and its non-fluid
 * force (N: gravity and contacts, e.g. psb_dem_forces) at the step's start;
 * mass is each particle's mass (kg). Every prediction of the step then also
 * predicts the boundary, x*_b = x_b + dt (v_b + dt (F_b + f_b) / m) with F_b
 * the fluid's reaction at the pressures of that prediction, and the density
 * passes see x*_b. After the step, psb_boundary_forces returns the F_b of the
 * last prediction: a DEM step given it as its external force moves the
 * spheres to that prediction (where no wall projects them). vel = NULL makes
 * the boundary static again; psb_set_boundary always does. No counterpart in
 * the reference, which has no fluid-solid coupling. */
int psb_set_boundary_motion(psb_ctx* ctx, const float* vel, const float* force, float mass);
/* DEM contexts: the force (N, n x 3 in particle-id order) the next step
 * would apply to each sphere apart from the external one: gravity and the
 * contacts at the current state (CudaSystem::update's force sum,
 * CudaSystem.cpp:226-245). Nothing moves. */
int psb_dem_forces(psb_ctx* ctx, float* force);
/* DEM contexts: an external force per sphere (N, n x 3 in particle-id
 * order) added to gravity and contacts in every step until replaced; NULL
 * removes it. Extends CudaSystem::update's force sum (CudaSystem.cpp:207-224),
 * which has gravity and contacts only. */
int psb_set_external_force(psb_ctx* ctx, const float* force);

/* Collision objects: the reference's ObjectCollision subclasses
 * (src/Kernel/Collision; Collision::collide, Collision.cpp:44-49), applied
 * in list order after each step's integrator and box walls, to the start
 * position, the new position and the new velocity (the half-step velocity
 * of the SPH systems, SphSystem.cpp:323-328; the velocity of DEM,
 * CudaSystem.cpp:253-257) before the velocity interpolation. Each object
 * follows its reference kernel as it executes:
 *  PLANE     PlaneCollision_Kernel.cu:7-81. v[0..11] corners A, B, C, D,
 *            v[12..14] normal N. A particle behind the plane and within the
 *            quad's extent on the axes N does not lie along goes to where
 *            its motion crossed the plane; the velocity loses (1 + r) of its
 *            normal part, r = elast |x - x_contact| / (dt |v|). A particle
 *            that did not move is left alone (the reference divides by 0).
 *  SPHERE    SphereCollision_Kernel.cu:7-91 through its launcher
 *            (SphereCollision.cu:9-16), which passes dt and the container
 *            flag in each other's place: the sphere (origin v[0..2], radius
 *            v[3]) always keeps particles inside it, and the restitution
 *            divides by 1 (container = 1) or 0 (container = 0, refused here
 *            when elast > 0: the reference's velocities become non-finite).
 *  CYLINDER  CylinderCollision_Kernel.cu:4-103: a container along the unit
 *            axis v[3..5] about v[0..2], radius v[6] less 0.04, length v[7],
 *            restitution 0.3 whatever elast says.
 *  MESH      MeshCollision_Kernel.cu:14-137: count faces, data = count x 12
 *            floats (A, B, C, N); the nearest face whose plane the particle
 *            is behind and whose triangle holds the contact point; elast is
 *            not used (0).
 *  HEIGHT    Linear/Gaussian/PeriodicHeightFieldCollision_Kernel.cu: inside
 *            the footprint v[0..2] (min) .. v[3..5] (max) in x and z, a
 *            particle below y = h(x, z) + min.y is lifted to it; normals by
 *            central differences (step 0.01). h is the sum of count terms,
 *            data = count x 6 floats {kind, c0, c1, c2, c3, c4}:
 *              PSB_HEIGHT_LINEAR    c0 x + c1 z
 *              PSB_HEIGHT_GAUSSIAN  c0 exp(-((x-c1)^2/(2 c3^2) + (z-c2)^2/(2 c4^2)))
 *              PSB_HEIGHT_COSINE    c0 cos(c1 (x cos c2 + z sin c2) + c3)
 *            One term gives the reference's linear or Gaussian field, cosine
 *            terms its periodic field, a mix its combined field (evaluated
 *            here at the new position; the reference evaluates a combined
 *            field at the start position).
 * Single-scene contexts, every method and profile. data is host memory,
 * copied. Replaces any earlier list; n = 0 removes it. */
#define PSB_MAX_COLLIDERS 32
#define PSB_MAX_COLLIDER_ITEMS 1048576      /* mesh faces or height terms per object */
enum {
    PSB_COLLIDER_PLANE = 1,
    PSB_COLLIDER_SPHERE = 2,
    PSB_COLLIDER_CYLINDER = 3,
    PSB_COLLIDER_MESH = 4,
    PSB_COLLIDER_HEIGHT = 5
};
enum { PSB_HEIGHT_LINEAR = 1, PSB_HEIGHT_GAUSSIAN = 2, PSB_HEIGHT_COSINE = 3 };
typedef struct psb_collider {
    int32_t type;        /* PSB_COLLIDER_* */
    int32_t container;   /* sphere: the reference's is_container */
    float elast;
    int32_t count;       /* mesh: faces; height: terms */
    float v[16];
    const float* data;   /* mesh faces or height terms (host) */
} psb_collider;
int psb_set_colliders(psb_ctx* ctx, const psb_collider* objs, int32_t n);

/* Emission mid-run (the reference's Emitters, src/Kernel/Emitters, and
 * PCI_SPHSystem::emitParticles / _initialize(begin, N),
 * PciSphSystem.cpp:50-160): particles appended at the end of the state
 * (ids n .. n + k - 1) before a step's neighbour search, into the capacity
 * the context was created with (the scene's n); nothing already resident
 * moves or crosses the host. Appended particles start with density and
 * pressure 0, the given velocity, and (SPH) a zero half-step velocity, as
 * the reference's SPHParticle constructor sets (SphParticle.cpp:33-34); a
 * DEM sphere's half-step velocity is its velocity. Single-scene contexts.
 *
 * psb_emit appends k particles from host arrays (vel, vel_half: NULL = 0);
 * PSB_EINVAL when n + k exceeds the capacity. */
int psb_emit(psb_ctx* ctx, int32_t k, const float* pos, const float* vel, const float* vel_half);

/* Emitters that run inside psb_step: at the start of every step, each
 * emitter whose emissions so far are fewer than `duration` appends one
 * emission (Emitters::emitParticles, Emitters.cpp:49-58, in the order the
 * emitters were added), all of them or none: a step whose emissions exceed
 * the capacity returns PSB_EINVAL before it changes anything. Each type
 * follows the reference's emitParticles:
 *  BOX        EmitterBox.cpp:29-47: float lattice from center - size/2 to
 *             center + size/2 (inclusive) in steps of 2 particle_radius, z
 *             outer, x inner, offset by world. v: center(3), size(3), world(3)
 *  SPHERE     EmitterSphere.cpp: rings of radius r = 0, rho, 2 rho, ... up
 *             to sqrt(radius^2 - y^2) (y absolute, as the reference), angle
 *             step acos(r / sqrt(r^2 + 2 rho^2)), layers y = center.y upward
 *             then below in steps of rho = particle_radius. v: center(3), radius
 *  CYLINDER   EmitterCylinder.cpp: the same rings up to the base radius,
 *             angle step acos(r / sqrt(r^2 + rho^2)), layers from P2.y to
 *             P1.y (P = center -/+ direction length/2). v: center(3),
 *             direction(3), base radius, length
 *  HEART      EmitterGirly.cpp: grid points of [-3, 3]^3 at 0.02 where
 *             |(x^2 + 2 y^2 + z^2 - 1)^3 - x^2 z^3| <= 0.001 (its 9/4 and 9/80
 *             are integer divisions)
 *  ELLIPSOID  EmitterElipsoide.cpp: `count` particles at center + (x + a cos t
 *             / 100, 0, z + b sin t / 100), x, z uniform in [-a/2, a/2],
 *             [-b/2, b/2], t uniform in [0, 2 pi). v: center(3), a, b
 *  MESH       EmitterMesh.cpp: per face, `count` particles at
 *             (u A + v B + w C)/(u + v + w), u, v, w uniform in [0, 0.5).
 *             data: n_faces x 9 floats (A, B, C), host memory, copied
 * The random emitters draw from SplitMix64 on (seed, emission, particle,
 * draw) in place of the reference's rand(). */
enum {
    PSB_EMITTER_BOX = 1,
    PSB_EMITTER_SPHERE = 2,
    PSB_EMITTER_CYLINDER = 3,
    PSB_EMITTER_HEART = 4,
    PSB_EMITTER_ELLIPSOID = 5,
    PSB_EMITTER_MESH = 6
};
#define PSB_MAX_EMITTERS 16
typedef struct psb_emitter {
    int32_t type;            /* PSB_EMITTER_* */
    int32_t duration;        /* emissions (the reference's durationTime) */
    int32_t count;           /* ellipsoid: per emission; mesh: per face */
    int32_t n_faces;         /* mesh */
    float particle_radius;   /* the emitting system's particle radius */
    float velocity[3];       /* velocityEmission */
    float v[12];
    const float* data;       /* mesh faces */
    uint64_t seed;           /* random emitters */
} psb_emitter;
int psb_add_emitter(psb_ctx* ctx, const psb_emitter* e);
/* Removes every emitter. */
int psb_clear_emitters(psb_ctx* ctx);
/* Host only (no context, no GPU): the positions emission number `emission`
 * of this emitter produces, in emission order, at most cap of them (out:
 * cap x 3 floats, may be NULL to count); *n receives the full count. The
 * random emitters use the same draws as the device. PSB_EINVAL (and
 * psb_add_emitter the same) for an emitter whose loops would not end (a
 * particle radius that is not positive, a value that is not finite, a step
 * below the float or double resolution of the coordinates it advances) or
 * whose emission could exceed 2^31 - 1 points; PSB_ENOMEM when the host
 * allocation fails. */
int psb_emitter_positions(const psb_emitter* e, int32_t emission, int64_t cap, float* out, int64_t* n);

/* The scene the context was created with (for a batch: scene 0 with n_max
 * the total), the particle count of the last upload (0 before one) and the
 * steps taken; psb_set_step_count overwrites the step count (checkpoints). */
int psb_context_info(const psb_ctx* ctx, psb_scene* scene, int32_t* n, int64_t* steps);
int psb_set_step_count(psb_ctx* ctx, int64_t steps);

/* ---- files --------------------------------------------------------------
 * The reference front end's export formats, so files made here open where
 * the reference's did. Numbers carry 9 significant digits (every float
 * exactly); the reference's writers round to 6. Paths are host file names;
 * each call returns PSB_EINVAL when the file cannot be written.
 * Txt particles, replacing ParticleExporter_Txt::_export for SPH systems
 * (ParticleExporter_Txt.cpp:27-33): "SPH <n>", then "-p x y z -m m -d rho"
 * per particle (pos: n x 3 doubles; density: n floats). */
int psb_write_txt(const char* path, int32_t n, const double* pos, double mass, const float* density);
/* XML particles, replacing ParticleExporter_XML::_export_SPHParticles
 * (ParticleExporter_XML.cpp:130-185): <Particles name="SPH System" dt count>,
 * <Gravity X Y Z Amp/>, and per particle the SPH attributes (mass, radius,
 * kernelParticles = its neighbour count, interactionRadius, restDensity,
 * gasStiffness, threshold, surfaceTension, viscosity) with <position>,
 * <velocity>, <velocityInterAv> (2 v - v+), <velocityInterAp> (v+) and
 * <color> (0, 0, 1). nbr_count may be NULL (written as 0). */
int psb_write_xml(const char* path, const psb_scene* scene, int32_t n, const double* pos, const double* vel,
                  const double* vel_half, const int32_t* nbr_count);
/* Mitsuba grid volume, replacing _exportData (UniformGrid.cu:266-300):
 * "VOL", version 3, encoding 1 (float32), resolution, 1 channel, the box
 * (bmin, bmax), then the field (dims[0] x dims[1] x dims[2] doubles, x
 * fastest, as psb_iso_field returns it) as floats. reference_layout = 0:
 * Mitsuba's order (x fastest); 1: the reference's file, which writes the z
 * resolution for all three axes and z fastest, for cubic grids only. */
int psb_write_vol(const char* path, const double* field, const int32_t dims[3], const float bmin[3], const float bmax[3],
                  int32_t reference_layout);
/* Wavefront OBJ of a triangle mesh (psb_extract_surface's output),
 * replacing SurfaceSPH::exportOBJ (SurfaceSPH.cpp:234-276): v lines, vn
 * lines (area-weighted vertex normals), then "f a//a b//b c//c" per
 * triangle. The reference also swaps y and z and scales for its renderer,
 * and skips the last triangle; these do neither. */
int psb_write_obj(const char* path, const float* vertices, int64_t n_vertices, const int32_t* triangles,
                  int64_t n_triangles);
/* The context's current state through the writers above (a download first). */
int psb_export_txt(psb_ctx* ctx, const char* path);
int psb_export_xml(psb_ctx* ctx, const char* path);
/* Checkpoints: the complete state a step continues from -- positions,
 * interpolated and half-step velocities, the carried pressure (read by the
 * warm starts), densities and the step count -- in particle-id order, with
 * the scene. Loading into a context of the same scene (any n_max large
 * enough) uploads it; stepping on gives bit for bit what the saved context
 * gives. Loading into a different scene returns PSB_EINVAL. No counterpart
 * in the reference, which restarts from its XML configuration only. */
int psb_checkpoint_save(psb_ctx* ctx, const char* path);
int psb_checkpoint_load(psb_ctx* ctx, const char* path);

/* FP64 diagnostics of the current state: with the corrector's convergence
 * reduction, the only FP64 arithmetic on the device. Each sum runs in FP64
 * in a fixed order (per-block partial sums, then one pass over the blocks),
 * so repeated calls give identical results. No counterpart in the reference.
 * n_out = 1: over all particles; n_out = the number of scenes of a batch:
 * one entry per scene. */
typedef struct psb_diag {
    double mass;                /* sum m */
    double momentum[3];         /* sum m v, v the interpolated velocity */
    double kinetic;             /* sum m |v|^2 / 2 */
    double potential;           /* sum -m g.x, g the step's gravity */
    double density_err_mean;    /* mean |rho - rho0| / rho0 over the last density pass */
    double density_err_max;     /* max of the same */
} psb_diag;
int psb_diagnostics(psb_ctx* ctx, psb_diag* out, int32_t n_out);

const char* psb_status_string(int32_t status);
const char* psb_last_error(const psb_ctx* ctx);
int32_t psb_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PSB_H */
