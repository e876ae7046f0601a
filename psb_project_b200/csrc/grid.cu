// grid.cu -- uniform-grid neighbour search: cell keys, stable radix sort by
// (cell, id), cell-ordered reindexing with cell ranges, neighbour lists.
//
// Replaces the reference's bucket grid (64 atomically filled slots per cell,
// src/Utils/Neighborhood/UniformGrid/UniformGridKernel.cu:30-55) and its
// 27-cell neighbour walk writing 200-slot lists (UniformGridKernel.cu:58-95).
// What stays identical, bit for bit:
//   * the cell index i = floor((x - Min)/sizeCell) in FP64 from the float
//     corner and cell edge (UniformGridKernel.cu:46-49), linearised as
//     i + j*nx + k*nx*ny (:50);
//   * the neighbour test length(x_i - x_j) <= h, self included (:81-82):
//     decided in FP32 with a guard band and, inside the band, re-evaluated
//     in FP64 with separately rounded operations in the reference's order.
// What differs by design: particles are sorted stably by (cell, id), so the
// neighbour order is deterministic; particles outside the grid are clamped
// into the border cells (the reference writes out of bounds there); lists
// are bounded (overflow raises a flag, never a trap).
#include "psb_internal.cuh"

namespace psb {

namespace {

__device__ __forceinline__ int cell_coord(float x, float corner, float cell, int dim, int& clamped) {
    const double t = floor(__ddiv_rn(__dsub_rn((double)x, (double)corner), (double)cell));
    if (!(t >= 0.0)) { clamped = 1; return 0; }          // also NaN
    if (t >= (double)dim) { clamped = 1; return dim - 1; }
    return (int)t;
}

// Clears the start entry of every cell the previous sort occupied.
__global__ void k_reset_cells(int n, const uint32_t* __restrict__ sorted_keys, uint32_t* __restrict__ cell_start) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t k = sorted_keys[s];
    if (s == 0 || sorted_keys[s - 1] != k) cell_start[k] = kEmpty;
}

// Cell key of every particle, written at its id so that a stable sort of
// the id-ordered keys yields (cell, id) order. A batch gives each scene its
// own grid and a block of keys after the previous scene's, so the sort keeps
// every scene in its own contiguous slot range, in the order it has alone.
template <bool BATCH>
__global__ void k_cell_keys(Params P, const float4* __restrict__ pos, const int* __restrict__ ids,
                            uint32_t* __restrict__ keys_by_id, uint32_t* __restrict__ slot_by_id,
                            int* __restrict__ clamped) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n) return;
    const float4 p = pos[s];
    const Grid g = BATCH ? P.scenes[P.slot_scene[s]].g : P.g;
    const uint32_t base = BATCH ? P.scenes[P.slot_scene[s]].cell_base : 0u;
    int c = 0;
    const int i = cell_coord(p.x, g.gx, g.cell, g.nx, c);
    const int j = cell_coord(p.y, g.gy, g.cell, g.ny, c);
    const int k = cell_coord(p.z, g.gz, g.cell, g.nz, c);
    const int id = ids[s];
    keys_by_id[id] = base + (uint32_t)i + (uint32_t)j * (uint32_t)g.nx + (uint32_t)k * (uint32_t)g.nx * (uint32_t)g.ny;
    slot_by_id[id] = (uint32_t)s;
    const unsigned ballot = __ballot_sync(__activemask(), c);
    if (ballot && (threadIdx.x & 31) == __ffs(ballot) - 1) atomicAdd(clamped, __popc(ballot));
}

// ---- LSD radix sort, 8-bit digits, three kernels per pass ----------------
constexpr int kItems = 8;                      // keys per thread per tile
constexpr int kTile = kBlock * kItems;         // 2048 keys per block

__global__ void k_radix_hist(int n, int shift, int nblocks, const uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const int i = base + r * kBlock + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Block-wide exclusive scan of one value per thread (blockDim == 256).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kBlock / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kBlock / 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kBlock / 32) s_warp[lane] = w;
    }
    __syncthreads();
    total = s_warp[kBlock / 32 - 1];
    const uint32_t before = warp ? s_warp[warp - 1] : 0u;
    __syncthreads();
    return before + x - v;
}

// Per-digit exclusive scan of the tiles' counts: block d scans hist[d][0..nb)
// in place and writes the digit's total.
__global__ void __launch_bounds__(kBlock) k_radix_scan(int nb, uint32_t* __restrict__ hist,
                                                       uint32_t* __restrict__ totals) {
    __shared__ uint32_t s_warp[kBlock / 32];
    uint32_t* h = hist + (size_t)blockIdx.x * nb;
    uint32_t carry = 0;
    for (int base = 0; base < nb; base += kBlock) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < nb ? h[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, s_warp, tot);
        if (i < nb) h[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Stable scatter. Tile items are ranked round by round (round r covers 256
// consecutive keys); inside a round, lanes holding the same digit are found
// with __match_any_sync and ranked by lane, warps by warp index.
__global__ void __launch_bounds__(kBlock) k_radix_scatter(int n, int shift, int nblocks,
                                                          const uint32_t* __restrict__ keys_in,
                                                          const uint32_t* __restrict__ vals_in,
                                                          uint32_t* __restrict__ keys_out,
                                                          uint32_t* __restrict__ vals_out,
                                                          const uint32_t* __restrict__ offsets,
                                                          const uint32_t* __restrict__ totals) {
    __shared__ uint32_t s_off[256];
    __shared__ uint32_t s_wc[kBlock / 32][256];
    __shared__ uint32_t s_warp[kBlock / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t all;
    const uint32_t digit_base = block_exclusive_scan(totals[tid], s_warp, all);
    s_off[tid] = digit_base + offsets[tid * nblocks + blockIdx.x];
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) s_wc[w][tid] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
    for (int r = 0; r < kItems; ++r) {
        const int i = base + r * kBlock + tid;
        const bool valid = i < n;
        const uint32_t key = valid ? keys_in[i] : 0u;
        const uint32_t val = valid ? vals_in[i] : 0u;
        const uint32_t d = valid ? ((key >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int wrank = __popc(peers & ((1u << lane) - 1u));
        if (valid && lane == __ffs(peers) - 1) s_wc[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t dst = s_off[d] + (uint32_t)wrank;
            for (int w = 0; w < warp; ++w) dst += s_wc[w][d];
            keys_out[dst] = key;
            vals_out[dst] = val;
        }
        __syncthreads();
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) { tot += s_wc[w][tid]; s_wc[w][tid] = 0; }
        s_off[tid] += tot;
        __syncthreads();
    }
}

// Gathers the particle state into sorted order and records each occupied
// cell's [start, end) slot range.
__global__ void k_reorder(int n, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                          const float4* __restrict__ pos, const float4* __restrict__ vel,
                          const float4* __restrict__ vap, const float2* __restrict__ rp, const int* __restrict__ ids,
                          float4* __restrict__ pos2, float4* __restrict__ vel2, float4* __restrict__ vap2,
                          float2* __restrict__ rp2, int* __restrict__ ids2, uint32_t* __restrict__ cell_start,
                          uint32_t* __restrict__ cell_end) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t s = vals[t];
    pos2[t] = pos[s];
    vel2[t] = vel[s];
    vap2[t] = vap[s];
    rp2[t] = rp[s];
    ids2[t] = ids[s];
    const uint32_t k = keys[t];
    if (t == 0 || keys[t - 1] != k) cell_start[k] = (uint32_t)t;
    if (t == n - 1 || keys[t + 1] != k) cell_end[k] = (uint32_t)t + 1u;
}

// The same in two launches, for the first step after an upload: positions,
// ids and cell ranges (all that the neighbour build reads) here, the rest
// in k_reorder_state once the upload's copies of it are in.
__global__ void k_reorder_pos(int n, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                              const float4* __restrict__ pos, const int* __restrict__ ids, float4* __restrict__ pos2,
                              int* __restrict__ ids2, uint32_t* __restrict__ cell_start,
                              uint32_t* __restrict__ cell_end) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t s = vals[t];
    pos2[t] = pos[s];
    ids2[t] = ids[s];
    const uint32_t k = keys[t];
    if (t == 0 || keys[t - 1] != k) cell_start[k] = (uint32_t)t;
    if (t == n - 1 || keys[t + 1] != k) cell_end[k] = (uint32_t)t + 1u;
}

// Gathers velocities, half-step velocities and (density, pressure) into
// sorted order.
__global__ void k_reorder_state(int n, const uint32_t* __restrict__ vals, const float4* __restrict__ vel,
                                const float4* __restrict__ vap, const float2* __restrict__ rp,
                                float4* __restrict__ vel2, float4* __restrict__ vap2, float2* __restrict__ rp2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t s = vals[t];
    vel2[t] = vel[s];
    vap2[t] = vap[s];
    rp2[t] = rp[s];
}

// Per-thread schedule: one thread per sorted particle. The three cells of a
// grid row are adjacent in sorted order, so each of the nine rows is one
// contiguous slot range; candidates are visited in increasing slot order and
// the list is sorted. In a batch the walk stays inside the particle's
// scene's grid.
template <bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_build_nbr(Params P, const float4* __restrict__ pos,
                                                  const uint32_t* __restrict__ keys,
                                                  const uint32_t* __restrict__ cell_start,
                                                  const uint32_t* __restrict__ cell_end, int* __restrict__ counts,
                                                  int* __restrict__ list, int* __restrict__ flags) {
    const int t = blockIdx.x * BS + threadIdx.x;
    const bool valid = t < P.n;       // every lane stays for the warp reductions below
    const int n = P.n;
    int cnt = 0;
    if (valid) {
        int* wq = list + nbr_index(0, n, t);
        const size_t qstride = (size_t)4 * (size_t)n;
        walk_neighbours<BATCH>(P, t, pos[t], pos, keys, cell_start, cell_end, [&](uint32_t q, float4) {
            // one 4-byte store per entry (buffering four in registers measured
            // slower); wq is entry cnt's quad, nbr_index(cnt, n, t) - (cnt & 3)
            if (cnt < P.cap) wq[cnt & 3] = (int)q;
            ++cnt;
            if ((cnt & 3) == 0 && cnt < P.cap) wq += qstride;
        });
        counts[t] = cnt;
        if (cnt > P.cap) atomicOr(&flags[0], 1);
    }
    nbr_flags(cnt, flags);
}

// Warp-cooperative schedule (row tiles). The lanes of a warp whose particles
// lie in the same grid row (same scene, j and k; consecutive sorted
// particles mostly do) form a group and walk its nine neighbour rows
// together. For each row the group's slot span -- the union of its lanes'
// three-cell ranges, one contiguous run of cells -- is staged 32 candidates
// at a time in shared memory, one coalesced load per lane, and each lane
// tests the staged candidates that lie inside its own range, in slot order.
// A lane therefore accepts the same candidates in the same order as in the
// per-thread schedule; the gathers become one load per candidate per group
// instead of one per candidate per lane.
template <bool BATCH, int BS>
__global__ void __launch_bounds__(BS) k_build_nbr_tile(Params P, const float4* __restrict__ pos,
                                                       const uint32_t* __restrict__ keys,
                                                       const uint32_t* __restrict__ cell_start,
                                                       const uint32_t* __restrict__ cell_end,
                                                       int* __restrict__ counts, int* __restrict__ list,
                                                       int* __restrict__ flags) {
    __shared__ float4 s_tile[BS];
    float4* tile = s_tile + (threadIdx.x & ~31u);
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * BS + threadIdx.x;
    const bool valid = t < P.n;
    const int n = P.n;
    int cnt = 0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int nx = 1, ny = 1, nz = 1, ci = 0, cj = 0, ck = 0;
    uint32_t base = 0, rowkey = kEmpty;     // rowkey: the global key of cell (0, j, k) of the particle's row
    if (valid) {
        const Grid g = BATCH ? P.scenes[P.slot_scene[t]].g : P.g;
        base = BATCH ? P.scenes[P.slot_scene[t]].cell_base : 0u;
        nx = g.nx; ny = g.ny; nz = g.nz;
        pi = pos[t];
        const uint32_t key = keys[t] - base;
        ci = (int)(key % (uint32_t)nx);
        cj = (int)((key / (uint32_t)nx) % (uint32_t)ny);
        ck = (int)(key / ((uint32_t)nx * (uint32_t)ny));
        rowkey = keys[t] - (uint32_t)ci;
    }
    const int a0 = max(ci - 1, 0), a1 = min(ci + 1, nx - 1);
    unsigned todo = __ballot_sync(0xffffffffu, valid);
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const uint32_t rk = __shfl_sync(0xffffffffu, rowkey, leader);
        const unsigned grp = __ballot_sync(0xffffffffu, valid && rowkey == rk);
        todo &= ~grp;
        const bool mine = (grp >> lane) & 1u;
        // the group shares scene, j, k and the grid: take them from the leader
        const int gj = __shfl_sync(0xffffffffu, cj, leader), gk = __shfl_sync(0xffffffffu, ck, leader);
        const int gnx = __shfl_sync(0xffffffffu, nx, leader), gny = __shfl_sync(0xffffffffu, ny, leader);
        const int gnz = __shfl_sync(0xffffffffu, nz, leader);
        const uint32_t gbase = __shfl_sync(0xffffffffu, base, leader);
        for (int k = max(gk - 1, 0); k <= min(gk + 1, gnz - 1); ++k) {
            for (int j = max(gj - 1, 0); j <= min(gj + 1, gny - 1); ++j) {
                const uint32_t row = gbase + (uint32_t)j * (uint32_t)gnx + (uint32_t)k * (uint32_t)gnx * (uint32_t)gny;
                uint32_t lo = kEmpty, hi = 0;
                if (mine) {
                    for (int a = a0; a <= a1; ++a) {
                        const uint32_t s = cell_start[row + a];
                        if (s != kEmpty) {
                            if (lo == kEmpty) lo = s;
                            hi = cell_end[row + a];
                        }
                    }
                }
                const uint32_t L = __reduce_min_sync(0xffffffffu, lo);
                const uint32_t H = __reduce_max_sync(0xffffffffu, hi);
                if (L == kEmpty) continue;
                for (uint32_t q0 = L; q0 < H; q0 += 32u) {
                    if (q0 + lane < H) tile[lane] = pos[q0 + lane];
                    __syncwarp();
                    if (mine && lo != kEmpty) {
                        // this lane's part of the staged chunk [q0, q0 + 32): [c0, c1)
                        const uint32_t c0 = lo > q0 ? lo - q0 : 0u;
                        const uint32_t c1 = hi > q0 ? min(hi - q0, 32u) : 0u;
                        for (uint32_t c = c0; c < c1; ++c) {
                            const float4 pj = tile[c];
                            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                            const float d2 = dist2(dx, dy, dz);
                            bool acc;
                            if (d2 < P.h2_lo) acc = true;
                            else if (d2 > P.h2_hi) acc = false;
                            else acc = exact_neighbor(pi, pj, P.h2_exact);
                            if (acc) {
                                if (cnt < P.cap) list[nbr_index(cnt, n, t)] = (int)(q0 + c);
                                ++cnt;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        }
    }
    if (valid) {
        counts[t] = cnt;
        if (cnt > P.cap) atomicOr(&flags[0], 1);
    }
    nbr_flags(cnt, flags);
}

inline int grid_of(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_reset_cells(cudaStream_t st, int n, const uint32_t* sorted_keys, uint32_t* cell_start) {
    if (n > 0) k_reset_cells<<<grid_of(n), kBlock, 0, st>>>(n, sorted_keys, cell_start);
}

void launch_cell_keys(cudaStream_t st, const Params& P, const float4* pos, const int* ids, uint32_t* keys_by_id,
                      uint32_t* slot_by_id, int* clamped) {
    if (P.n <= 0) return;
    if (P.scenes) k_cell_keys<true><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, ids, keys_by_id, slot_by_id, clamped);
    else k_cell_keys<false><<<grid_of(P.n), kBlock, 0, st>>>(P, pos, ids, keys_by_id, slot_by_id, clamped);
}

int radix_blocks(int n) { return (n + kTile - 1) / kTile; }

int radix_sort(cudaStream_t st, int n, int bits, uint32_t* keys[2], uint32_t* vals[2], uint32_t* hist, int nblocks_cap) {
    const int nb = radix_blocks(n);
    if (nb > nblocks_cap || n <= 0) return 0;
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        k_radix_hist<<<nb, kBlock, 0, st>>>(n, shift, nb, keys[cur], hist);
        k_radix_scan<<<256, kBlock, 0, st>>>(nb, hist, hist + (size_t)256 * nb);
        k_radix_scatter<<<nb, kBlock, 0, st>>>(n, shift, nb, keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], hist,
                                               hist + (size_t)256 * nb);
        cur ^= 1;
    }
    return cur;
}

void launch_reorder(cudaStream_t st, int n, const uint32_t* keys, const uint32_t* vals, const float4* pos,
                    const float4* vel, const float4* vap, const float2* rp, const int* ids, float4* pos2, float4* vel2,
                    float4* vap2, float2* rp2, int* ids2, uint32_t* cell_start, uint32_t* cell_end) {
    if (n > 0)
        k_reorder<<<grid_of(n), kBlock, 0, st>>>(n, keys, vals, pos, vel, vap, rp, ids, pos2, vel2, vap2, rp2, ids2,
                                                 cell_start, cell_end);
}

void launch_reorder_pos(cudaStream_t st, int n, const uint32_t* keys, const uint32_t* vals, const float4* pos,
                        const int* ids, float4* pos2, int* ids2, uint32_t* cell_start, uint32_t* cell_end) {
    if (n > 0)
        k_reorder_pos<<<grid_of(n), kBlock, 0, st>>>(n, keys, vals, pos, ids, pos2, ids2, cell_start, cell_end);
}

void launch_reorder_state(cudaStream_t st, int n, const uint32_t* vals, const float4* vel, const float4* vap,
                          const float2* rp, float4* vel2, float4* vap2, float2* rp2) {
    if (n > 0) k_reorder_state<<<grid_of(n), kBlock, 0, st>>>(n, vals, vel, vap, rp, vel2, vap2, rp2);
}

void launch_build_nbr(cudaStream_t st, const Params& P, const float4* pos, const uint32_t* keys,
                      const uint32_t* cell_start, const uint32_t* cell_end, int* counts, int* list, int* flags) {
    if (P.n <= 0) return;
    with_block(P.tune.nbr_block, [&](auto B) {
        constexpr int BS = decltype(B)::value;
        const unsigned g = (unsigned)((P.n + BS - 1) / BS);
        auto go = [&](auto kernel) { kernel<<<g, BS, 0, st>>>(P, pos, keys, cell_start, cell_end, counts, list, flags); };
        if (P.tune.nbr_schedule == 1) {
            if (P.scenes) go(k_build_nbr_tile<true, BS>); else go(k_build_nbr_tile<false, BS>);
        } else {
            if (P.scenes) go(k_build_nbr<true, BS>); else go(k_build_nbr<false, BS>);
        }
    });
}

}  // namespace psb
