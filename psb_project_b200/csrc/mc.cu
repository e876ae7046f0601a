// mc.cu -- iso field on a node grid and marching-cubes surface extraction.
//
// Iso field (one thread per node, gathered over the particle grid's cell
// rings, FP64 accumulation):
//   reference profile: evaluateIso_Kernel (UniformGridKernel.cu:98-138):
//     r = h / scale, ring = floor(1/scale) cells,
//     iso(x) = sum_{|x - x_j| <= r} (1/r^6) (r^2 - d^2)^3, each term in float
//     as the reference's powf computes it;
//   config profile: the density-based colour field
//     c(x) = sum_j (m / rho_j) W_poly6(|x - x_j|, h), ring = 1 cell.
//
// Marching cubes (polygonize_MarchingCube_Kernel, MarchingCube_Kernel.cu:36-
// 160): corners and edges numbered as there, case bit c set when
// iso(corner c) <= level, vertices on the edges by linear interpolation with
// the reference's 1e-6 guards. The reference keeps 15 vertex slots per cell
// and welds vertices on the host in O(V^2) (SurfaceSPH.cpp:120-186); here
// every active grid edge owns one vertex (its index is the edge's rank in an
// exclusive scan), so the mesh is welded by construction, and triangles are
// written compacted through a second scan.
//
// The triangle table is generated here, not copied: for each of the 256
// cases the active edges of every cube face are joined into segments (a face
// with four active edges separates its two set corners), the segments close
// into loops on the cube surface, each loop is oriented so that its normal
// points toward the set corners (iso <= level, the outside of a fluid) and
// fanned into triangles. The face rule depends only on the face's four
// corners, so neighbouring cubes agree on every shared face and the surface
// is closed wherever the field is.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <vector>

#include "psb_internal.cuh"

namespace psb {

namespace {

// Corner c at (x, y, z) offsets; edges as corner pairs (the reference's numbering).
#define PSB_MC_CORNERS {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}}
#define PSB_MC_EDGES {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}}
constexpr int kCorner[8][3] = PSB_MC_CORNERS;
constexpr int kEdge[12][2] = PSB_MC_EDGES;
constexpr int kFace[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 3, 7, 4}, {1, 2, 6, 5}, {0, 1, 5, 4}, {3, 2, 6, 7}};
__constant__ int c_corner[8][3] = PSB_MC_CORNERS;
__constant__ int c_edge[12][2] = PSB_MC_EDGES;

__constant__ int8_t c_tri[256][kMcMaxTri * 3];
__constant__ uint8_t c_ntri[256];

int edge_of(int a, int b) {
    for (int e = 0; e < 12; ++e)
        if ((kEdge[e][0] == a && kEdge[e][1] == b) || (kEdge[e][0] == b && kEdge[e][1] == a)) return e;
    return -1;
}

}  // namespace

void mc_build_table(uint8_t ntri[256], int8_t tri[256][kMcMaxTri * 3]) {
    for (int cs = 0; cs < 256; ++cs) {
        ntri[cs] = 0;
        std::memset(tri[cs], -1, kMcMaxTri * 3);
        auto set = [&](int c) { return (cs >> c) & 1; };
        int link[12][2];
        int deg[12] = {0};
        auto join = [&](int e0, int e1) {
            link[e0][deg[e0]++] = e1;
            link[e1][deg[e1]++] = e0;
        };
        for (int f = 0; f < 6; ++f) {
            const int* q = kFace[f];
            int act[4], na = 0;
            for (int k = 0; k < 4; ++k) {
                const int a = q[k], b = q[(k + 1) & 3];
                if (set(a) != set(b)) act[na++] = edge_of(a, b);
            }
            if (na == 2) {
                join(act[0], act[1]);
            } else if (na == 4) {          // separate each set corner from the rest
                for (int k = 0; k < 4; ++k) {
                    if (!set(q[k])) continue;
                    join(edge_of(q[(k + 3) & 3], q[k]), edge_of(q[k], q[(k + 1) & 3]));
                }
            }
        }
        bool used[12] = {false};
        int nt = 0;
        for (int start = 0; start < 12; ++start) {
            if (deg[start] != 2 || used[start]) continue;
            int loop[12], nl = 0, prev = -1, cur = start;
            do {
                loop[nl++] = cur;
                used[cur] = true;
                const int nxt = link[cur][0] != prev ? link[cur][0] : link[cur][1];
                prev = cur;
                cur = nxt;
            } while (cur != start && nl < 12);
            // orientation: Newell normal of the edge-midpoint polygon against
            // the direction from unset to set corners across the loop's edges
            double nrm[3] = {0, 0, 0}, dir[3] = {0, 0, 0};
            double mid[12][3];
            for (int k = 0; k < nl; ++k) {
                const int a = kEdge[loop[k]][0], b = kEdge[loop[k]][1];
                for (int d = 0; d < 3; ++d) mid[k][d] = 0.5 * (kCorner[a][d] + kCorner[b][d]);
                const int s = set(a) ? a : b, u = set(a) ? b : a;
                for (int d = 0; d < 3; ++d) dir[d] += kCorner[s][d] - kCorner[u][d];
            }
            for (int k = 0; k < nl; ++k) {
                const double* p = mid[k];
                const double* r = mid[(k + 1) % nl];
                nrm[0] += (p[1] - r[1]) * (p[2] + r[2]);
                nrm[1] += (p[2] - r[2]) * (p[0] + r[0]);
                nrm[2] += (p[0] - r[0]) * (p[1] + r[1]);
            }
            const bool flip = nrm[0] * dir[0] + nrm[1] * dir[1] + nrm[2] * dir[2] < 0;
            for (int k = 1; k + 1 < nl; ++k) {
                int v0 = loop[0], v1 = loop[k], v2 = loop[k + 1];
                if (flip) { const int t = v1; v1 = v2; v2 = t; }
                tri[cs][3 * nt + 0] = (int8_t)v0;
                tri[cs][3 * nt + 1] = (int8_t)v1;
                tri[cs][3 * nt + 2] = (int8_t)v2;
                ++nt;
            }
        }
        ntri[cs] = (uint8_t)nt;
    }
}

namespace {

// ---- iso field ----------------------------------------------------------------
template <bool REF>
__global__ void k_iso_field(IsoParams Q, Params P, const float4* __restrict__ pos, const float2* __restrict__ rp,
                            const uint32_t* __restrict__ cell_start, const uint32_t* __restrict__ cell_end,
                            double* __restrict__ iso) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (node >= nn) return;
    const int ix = (int)(node % Q.dims[0]);
    const int iy = (int)((node / Q.dims[0]) % Q.dims[1]);
    const int iz = (int)(node / ((long long)Q.dims[0] * Q.dims[1]));
    const double px = Q.origin[0] + ix * Q.spacing[0];
    const double py = Q.origin[1] + iy * Q.spacing[1];
    const double pz = Q.origin[2] + iz * Q.spacing[2];
    // particle-grid cell of the node, as the reference computes it
    const int I = (int)floor((px - (double)P.g.gx) / (double)P.g.cell);
    const int J = (int)floor((py - (double)P.g.gy) / (double)P.g.cell);
    const int K = (int)floor((pz - (double)P.g.gz) / (double)P.g.cell);
    const int ring = Q.ring;
    double acc = 0.0;
    for (int i = I - ring; i <= I + ring; ++i) {
        if (i < 0 || i >= P.g.nx) continue;
        for (int j = J - ring; j <= J + ring; ++j) {
            if (j < 0 || j >= P.g.ny) continue;
            for (int k = K - ring; k <= K + ring; ++k) {
                if (k < 0 || k >= P.g.nz) continue;
                const uint32_t c = (uint32_t)i + (uint32_t)j * P.g.nx + (uint32_t)k * P.g.nx * P.g.ny;
                const uint32_t s = cell_start[c];
                if (s == kEmpty) continue;
                const uint32_t e = cell_end[c];
                for (uint32_t t = s; t < e; ++t) {
                    const float4 x = pos[t];
                    const double dx = px - x.x, dy = py - x.y, dz = pz - x.z;
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    if (REF) {
                        // d = length(pos1 - pos2); (1/powf(r,6)) * powf(r*r - d*d, 3) in float
                        const double d = sqrt(d2);
                        if (!(d <= Q.r)) continue;
                        const float term = (1.f / powf((float)Q.r, 6.f)) * powf((float)(Q.r * Q.r - d * d), 3.f);
                        acc += (double)term;
                    } else {
                        const double q = d2 * Q.inv_r2;
                        if (q >= 1.0) continue;
                        const double w = 1.0 - q;
                        acc += Q.k_colour * (w * w * w) / (double)rp[t].x;
                    }
                }
            }
        }
    }
    iso[node] = acc;
}

// ---- marching cubes -----------------------------------------------------------
__device__ __forceinline__ int cube_case(const IsoParams& Q, const double* __restrict__ iso, int x, int y, int z) {
    const long long sx = 1, sy = Q.dims[0], sz = (long long)Q.dims[0] * Q.dims[1];
    const long long b = x + y * sy + z * sz;
    int cs = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const long long o = b + c_corner[c][0] * sx + c_corner[c][1] * sy + c_corner[c][2] * sz;
        if (iso[o] <= Q.level) cs |= 1 << c;
    }
    return cs;
}

__device__ __forceinline__ bool edge_active(const IsoParams& Q, const double* __restrict__ iso, long long node,
                                            int axis, int x, int y, int z) {
    const int c = axis == 0 ? x : (axis == 1 ? y : z);
    if (c + 1 >= Q.dims[axis]) return false;
    const long long step = axis == 0 ? 1 : (axis == 1 ? Q.dims[0] : (long long)Q.dims[0] * Q.dims[1]);
    return (iso[node] <= Q.level) != (iso[node + step] <= Q.level);
}

// Per cube (indexed by its lowest node): triangle count. Per node: 0/1 for
// each of its +x, +y, +z edges crossing the level. Both arrays carry one
// trailing zero so that their in-place exclusive scans end in the totals.
__global__ void k_mc_classify(IsoParams Q, const double* __restrict__ iso, uint32_t* __restrict__ cube_tris,
                              uint32_t* __restrict__ edge_flag) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (node == nn) { cube_tris[nn] = 0; edge_flag[3 * nn] = 0; }
    if (node >= nn) return;
    const int x = (int)(node % Q.dims[0]);
    const int y = (int)((node / Q.dims[0]) % Q.dims[1]);
    const int z = (int)(node / ((long long)Q.dims[0] * Q.dims[1]));
#pragma unroll
    for (int a = 0; a < 3; ++a) edge_flag[3 * node + a] = edge_active(Q, iso, node, a, x, y, z) ? 1u : 0u;
    uint32_t nt = 0;
    if (x + 1 < Q.dims[0] && y + 1 < Q.dims[1] && z + 1 < Q.dims[2]) nt = c_ntri[cube_case(Q, iso, x, y, z)];
    cube_tris[node] = nt;
}

// Global edge id (node * 3 + axis) of cube edge e of the cube at (x, y, z).
__device__ __forceinline__ long long global_edge(const IsoParams& Q, int x, int y, int z, int e) {
    const int a = c_edge[e][0], b = c_edge[e][1];
    const int lo = (c_corner[a][0] + c_corner[a][1] + c_corner[a][2]) <= (c_corner[b][0] + c_corner[b][1] + c_corner[b][2]) ? a : b;
    const int hi = lo == a ? b : a;
    const int axis = c_corner[hi][0] != c_corner[lo][0] ? 0 : (c_corner[hi][1] != c_corner[lo][1] ? 1 : 2);
    const long long nx = x + c_corner[lo][0], ny = y + c_corner[lo][1], nz = z + c_corner[lo][2];
    return 3 * (nx + ny * Q.dims[0] + nz * (long long)Q.dims[0] * Q.dims[1]) + axis;
}

// vertexInterpolate_MarchingCube (MarchingCube_Kernel.cu:143-155)
__device__ __forceinline__ double interp(double level, double v1, double v2, double p1, double p2) {
    if (fabs(level - v1) < 0.000001) return p1;
    if (fabs(level - v2) < 0.000001) return p2;
    if (fabs(v1 - v2) < 0.000001) return p1;
    const double mu = (level - v1) / (v2 - v1);
    return p1 + mu * (p2 - p1);
}

__global__ void k_mc_vertices(IsoParams Q, const double* __restrict__ iso, const uint32_t* __restrict__ edge_off,
                              float* __restrict__ vert) {
    const long long ge = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (ge >= 3 * nn) return;
    const long long node = ge / 3;
    const int axis = (int)(ge % 3);
    const int x = (int)(node % Q.dims[0]);
    const int y = (int)((node / Q.dims[0]) % Q.dims[1]);
    const int z = (int)(node / ((long long)Q.dims[0] * Q.dims[1]));
    if (!edge_active(Q, iso, node, axis, x, y, z)) return;
    const long long step = axis == 0 ? 1 : (axis == 1 ? Q.dims[0] : (long long)Q.dims[0] * Q.dims[1]);
    const double v1 = iso[node], v2 = iso[node + step];
    const double p[3] = {Q.origin[0] + x * Q.spacing[0], Q.origin[1] + y * Q.spacing[1], Q.origin[2] + z * Q.spacing[2]};
    const uint32_t o = edge_off[ge];
    for (int d = 0; d < 3; ++d) {
        const double q = d == axis ? p[d] + Q.spacing[d] : p[d];
        vert[3 * (size_t)o + d] = (float)interp(Q.level, v1, v2, p[d], q);
    }
}

__global__ void k_mc_triangles(IsoParams Q, const double* __restrict__ iso, const uint32_t* __restrict__ tri_off,
                               const uint32_t* __restrict__ edge_off, int32_t* __restrict__ tris) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (node >= nn) return;
    const int x = (int)(node % Q.dims[0]);
    const int y = (int)((node / Q.dims[0]) % Q.dims[1]);
    const int z = (int)(node / ((long long)Q.dims[0] * Q.dims[1]));
    if (x + 1 >= Q.dims[0] || y + 1 >= Q.dims[1] || z + 1 >= Q.dims[2]) return;
    const int cs = cube_case(Q, iso, x, y, z);
    const uint32_t base = tri_off[node];
    const int nt = c_ntri[cs];
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k)
            tris[3 * ((size_t)base + t) + k] = (int32_t)edge_off[global_edge(Q, x, y, z, c_tri[cs][3 * t + k])];
}

// polygonize_MarchingCube_Kernel (MarchingCube_Kernel.cu:36-139) on the
// reference's layout: nodes are double4 (x, y, z, value); every cube with a
// triangle appends its triangles' vertices, three per triangle, to its own
// `slots` vertex slots (vertex[c * slots + k], index[c * slots + k] = k) and
// counts them in count[c], which it reads first (the reference accumulates).
// Vertices are interpolated on the cube's edges in the reference's corner
// order; a cube whose slots would overflow stops and raises *overflow.
__global__ void k_mc_polygonize_slots(const double* __restrict__ node4, int nx, int ny, int nz, double level,
                                      int* __restrict__ count, double* __restrict__ vertex, int* __restrict__ index,
                                      int slots, int* __restrict__ overflow) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)nx * ny * nz) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
    if (x + 1 >= nx || y + 1 >= ny || z + 1 >= nz) return;
    long long corner[8];
    int cs = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        corner[k] = (x + c_corner[k][0]) + (long long)(y + c_corner[k][1]) * nx +
                    (long long)(z + c_corner[k][2]) * nx * ny;
        if (node4[4 * corner[k] + 3] <= level) cs |= 1 << k;
    }
    const int nt = c_ntri[cs];
    if (nt == 0) return;
    int m = count[c];
    for (int t = 0; t < nt; ++t)
        for (int v = 0; v < 3; ++v) {
            if (m < 0 || m >= slots) { *overflow = 1; count[c] = m; return; }
            const int e = c_tri[cs][3 * t + v];
            const long long a = corner[c_edge[e][0]], b = corner[c_edge[e][1]];
            const double va = node4[4 * a + 3], vb = node4[4 * b + 3];
            double* out = vertex + 3 * ((size_t)c * slots + m);
            for (int d = 0; d < 3; ++d) out[d] = interp(level, va, vb, node4[4 * a + d], node4[4 * b + d]);
            index[(size_t)c * slots + m] = m;
            ++m;
        }
    count[c] = m;
}

// ---- exclusive scan of uint32 (three-level, 1024 items per block) ------------
constexpr int kScanThreads = 256, kScanItems = 4, kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(long long n, uint32_t* __restrict__ data,
                                                             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t s[kScanThreads];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], tot = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? data[base + k] : 0u;
        tot += v[k];
    }
    s[threadIdx.x] = tot;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {     // Hillis-Steele over the thread totals
        const uint32_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t run = s[threadIdx.x] - tot;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) data[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1 && tile_sums) tile_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_add(long long n, uint32_t* __restrict__ data, const uint32_t* __restrict__ tile_offsets) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) data[i] += tile_offsets[i / kScanTile];
}

inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_mc_polygonize_slots(cudaStream_t st, const double* node4, int nx, int ny, int nz, double level, int* count,
                                double* vertex, int* index, int slots) {
    static int* d_overflow = nullptr;
    if (!d_overflow && cudaMalloc((void**)&d_overflow, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        d_overflow = nullptr;
    }
    int* flag = d_overflow;
    if (!flag) return;
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    const long long nn = (long long)nx * ny * nz;
    k_mc_polygonize_slots<<<blocks_for(nn, 256), 256, 0, st>>>(node4, nx, ny, nz, level, count, vertex, index, slots,
                                                               flag);
    int h = 0;
    cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if (h) std::fprintf(stderr, "polygonize_MarchingCube_CUDA: a cell needed more than %d vertex slots (stopped there)\n",
                        slots);
}

void mc_upload_table(cudaStream_t st) {
    static uint8_t ntri[256];
    static int8_t tri[256][kMcMaxTri * 3];
    static bool built = false;
    if (!built) {
        mc_build_table(ntri, tri);
        built = true;
    }
    cudaMemcpyToSymbolAsync(c_ntri, ntri, sizeof(ntri), 0, cudaMemcpyHostToDevice, st);
    cudaMemcpyToSymbolAsync(c_tri, tri, sizeof(tri), 0, cudaMemcpyHostToDevice, st);
}

long long scan_scratch_words(long long n) {
    const long long t1 = (n + kScanTile - 1) / kScanTile;
    const long long t2 = (t1 + kScanTile - 1) / kScanTile;
    return t1 + t2 + 1;
}

void scan_exclusive_u32(cudaStream_t st, long long n, uint32_t* data, uint32_t* scratch) {
    if (n <= 0) return;
    const long long t1 = (n + kScanTile - 1) / kScanTile;
    uint32_t* s1 = scratch;
    uint32_t* s2 = scratch + t1;
    k_scan_tiles<<<(unsigned)t1, kScanThreads, 0, st>>>(n, data, s1);
    if (t1 > 1) {
        const long long t2 = (t1 + kScanTile - 1) / kScanTile;
        k_scan_tiles<<<(unsigned)t2, kScanThreads, 0, st>>>(t1, s1, s2);
        if (t2 > 1) {   // t2 <= kScanTile while n < 2^30
            k_scan_tiles<<<1, kScanThreads, 0, st>>>(t2, s2, nullptr);
            k_scan_add<<<blocks_for(t1, 256), 256, 0, st>>>(t1, s1, s2);
        }
        k_scan_add<<<blocks_for(n, 256), 256, 0, st>>>(n, data, s1);
    }
}

void launch_iso_field(cudaStream_t st, const IsoParams& Q, const Params& P, const float4* pos, const float2* rp,
                      const uint32_t* cell_start, const uint32_t* cell_end, double* iso) {
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    if (nn <= 0) return;
    if (P.ref) k_iso_field<true><<<blocks_for(nn, 256), 256, 0, st>>>(Q, P, pos, rp, cell_start, cell_end, iso);
    else k_iso_field<false><<<blocks_for(nn, 256), 256, 0, st>>>(Q, P, pos, rp, cell_start, cell_end, iso);
}

void launch_mc_classify(cudaStream_t st, const IsoParams& Q, const double* iso, uint32_t* cube_tris,
                        uint32_t* edge_flag) {
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    k_mc_classify<<<blocks_for(nn + 1, 256), 256, 0, st>>>(Q, iso, cube_tris, edge_flag);
}

void launch_mc_emit(cudaStream_t st, const IsoParams& Q, const double* iso, const uint32_t* edge_off,
                    const uint32_t* tri_off, float* vert, int32_t* tris) {
    const long long nn = (long long)Q.dims[0] * Q.dims[1] * Q.dims[2];
    k_mc_vertices<<<blocks_for(3 * nn, 256), 256, 0, st>>>(Q, iso, edge_off, vert);
    k_mc_triangles<<<blocks_for(nn, 256), 256, 0, st>>>(Q, iso, tri_off, edge_off, tris);
}

}  // namespace psb
