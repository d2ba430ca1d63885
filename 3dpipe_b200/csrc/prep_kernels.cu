// prep_kernels.cu -- GPU LOD preparation (tdp_raw_from_meshes): LOD-100 meshes
// in, a RAW tile out, with every step of the preparation on the device.
//
// Replaces the reference's CGAL preparation of its tiles: progressive
// decimation into LODs (src/spatial/himesh_comp.cpp:28-190), skeleton voxels
// (src/spatial/himesh_skeleton.cpp:17-168), LOD triangles to voxels
// (src/spatial/himesh_retrieve.cpp:183-200), the per-triangle Hausdorff bounds
// (src/spatial/himesh_hausdorff.cpp:197-296, done here by
// tdp_tile_compute_bounds) and the RAW writer (src/storage/tile_IO.cpp:79-172).
// The rule, per object with vertices P (float, evaluated in double) and
// LOD-100 facets F[0..m):
//  1. LODs 80, 60, 40, 20 by half-edge collapse, shortest edge first, keyed
//     (|P_a - P_b|^2, a, b) with a < b.  The smallest key among the candidate
//     edges is tried: a into b, else b into a, each refused unless exactly two
//     live facets hold both (third vertices w1 != w2), the common neighbours of
//     the two are exactly {w1, w2}, w1 and w2 have more than 3 neighbours each,
//     and no facet of the removed vertex turns (normal n0 -> n1:
//     |n1| >= 1e-12 (|n0| + 1e-300) and n0.n1 >= 0.3 |n0||n1|).  A refused edge
//     stops being a candidate until a collapse changes one of its ends; every
//     edge of the kept vertex becomes a candidate again after a collapse.  A LOD
//     is the live facets in index order once their count is <= floor(m l / 100)
//     (or no candidate is left).  This is the sequential priority-queue
//     decimation with versioned entries restated without the queue: the
//     candidate set is exactly the queue's set of current entries.
//  2. nseed = m / voxel_size + 1 farthest-point seeds from vertex 0, two Lloyd
//     steps (sums in vertex order), each facet to the seed nearest its
//     barycentre, a seed's core = vertex 0 of its nearest facet.
//  3. LOD-100 triangles to the voxel with the nearest core by first vertex;
//     voxels left without a LOD-100 triangle are dropped; then every LOD is
//     assigned the same way to the voxels kept, triangles keeping LOD order.
//  4. Transform = the vertex nearest the centre of the float bounding box.
// Ties go to the lowest index everywhere.  Work layout: one CTA per object.
// Decimation keeps the object's facets (16- or 32-bit vertex ids), flags and
// four vertex bitmasks in shared memory (global memory for objects too large
// for it); each thread owns the facets tid + k T, caches the smallest key of
// its own candidate edges and recomputes it only after one of its facets
// changed; a round is a block argmin, one scan of the facets around the edge
// (links, neighbour masks, normals) and one applying scan.  This file is built
// with -fmad=false: every product and sum is rounded on its own, as on the host.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "storage/dt_format.h"

namespace tdp {
namespace {

constexpr int kDecLods = kNumLods - 1;  // LODs made by decimation (20..80)
constexpr int kPrepThreads = 256;       // voxel and writer kernels
constexpr size_t kSmemSmall = 40 << 10;  // decimation in shared memory, 128 threads
constexpr size_t kSmemLarge = 200 << 10; // decimation in shared memory, 1024 threads

struct Meshes {  // one batch on the device; object o: vertices V[3 voff[o]..), facets F[3 foff[o]..)
    const float* V;
    const int64_t* voff;
    const uint32_t* F;
    const int64_t* foff;
    int n;
};

struct VoxScratch {
    double* dmin;      // per vertex
    uint32_t* asg;     // per vertex
    double* seed;      // 3 per seed
    unsigned long long* bestd;  // per seed
    uint32_t* bestf;   // per seed
    uint32_t* core;    // per seed (kept voxels first)
    uint32_t* nvox;    // per object
    uint32_t* tvox;    // kNumLods planes of Ftot: voxel of each LOD triangle
    uint32_t* ord;     // kNumLods planes of Ftot: LOD triangles grouped by voxel
    uint32_t* vcnt;    // kNumLods planes of Stot: triangles per voxel
    uint32_t* vst;     // kNumLods planes of Stot: first grouped index per voxel
    const int64_t* soff;  // per object: first seed
    int64_t Ftot, Stot;
};

__host__ __device__ inline size_t round16(size_t x) { return (x + 15) & ~(size_t)15; }

__device__ __forceinline__ double3 vtx(const float* P, uint32_t i) {
    return make_double3((double)P[3 * (size_t)i], (double)P[3 * (size_t)i + 1], (double)P[3 * (size_t)i + 2]);
}
__device__ __forceinline__ double dist2(double3 a, double3 b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz;
}
__device__ __forceinline__ double3 sub3(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ bool key_less(double l1, uint32_t a1, uint32_t b1, double l2, uint32_t a2, uint32_t b2) {
    if (l1 != l2) return l1 < l2;
    if (a1 != a2) return a1 < a2;
    return b1 < b2;
}

// true when replacing u by v turns facet (x, y, z) (which holds u, not v)
__device__ bool turns(const float* P, uint32_t x, uint32_t y, uint32_t z, uint32_t u, uint32_t v) {
    const double3 p0 = vtx(P, x), p1 = vtx(P, y), p2 = vtx(P, z);
    const double3 q0 = vtx(P, x == u ? v : x), q1 = vtx(P, y == u ? v : y), q2 = vtx(P, z == u ? v : z);
    const double3 n0 = cross3(sub3(p1, p0), sub3(p2, p0)), n1 = cross3(sub3(q1, q0), sub3(q2, q0));
    const double a0 = sqrt(dot3(n0, n0)), a1 = sqrt(dot3(n1, n1));
    return a1 < 1e-12 * (a0 + 1e-300) || dot3(n0, n1) < 0.3 * a0 * a1;
}

__device__ __forceinline__ void mark(uint32_t* M, uint32_t x, uint32_t y, uint32_t z, uint32_t c) {
    if (x != c) atomicOr(M + (x >> 5), 1u << (x & 31));
    if (y != c) atomicOr(M + (y >> 5), 1u << (y & 31));
    if (z != c) atomicOr(M + (z >> 5), 1u << (z & 31));
}

// smallest key (|P_a - P_b|^2, a, b) over the candidate slots of facet f with
// flags fla, folded into (bl, ba, bb, bf)
template <typename VI>
__device__ __forceinline__ void fold_facet(const float* P, const VI* fv, uint32_t f, uint32_t fla, double& bl,
                                           uint32_t& ba, uint32_t& bb, uint32_t& bf) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        if (fla & (2u << j)) continue;
        const uint32_t x = fv[3 * f + j], y = fv[3 * f + (j == 2 ? 0 : j + 1)];
        const uint32_t a = min(x, y), b = max(x, y);
        const double L = dist2(vtx(P, a), vtx(P, b));
        if (key_less(L, a, b, bl, ba, bb)) { bl = L; ba = a; bb = b; bf = f; }
    }
}

// bytes of decimation storage for an object (facets, flags, 4 masks)
__host__ __device__ inline size_t dec_bytes(int64_t n, int64_t m, size_t vi) {
    return round16(3 * (size_t)m * vi) + round16((size_t)m) + 16 * (size_t)((n + 31) / 32);
}

// ------------------------------------------------------------------ validation
// first object (lowest index) without vertices or facets, with a vertex index
// out of range, a facet repeating a vertex, or a non-finite coordinate
__global__ void k_validate(Meshes M, int* first_bad) {
    for (int o = blockIdx.x; o < M.n; o += gridDim.x) {
        const int64_t v0 = M.voff[o], v1 = M.voff[o + 1], f0 = M.foff[o], f1 = M.foff[o + 1];
        bool bad = v1 <= v0 || f1 <= f0 || v1 - v0 > 0xffffffffLL;
        const uint64_t n = (uint64_t)(v1 - v0);
        for (int64_t f = f0 + threadIdx.x; !bad && f < f1; f += blockDim.x) {
            const uint32_t a = M.F[3 * f], b = M.F[3 * f + 1], c = M.F[3 * f + 2];
            bad = a >= n || b >= n || c >= n || a == b || b == c || a == c;
        }
        for (int64_t i = 3 * v0 + threadIdx.x; !bad && i < 3 * v1; i += blockDim.x) bad = !isfinite(M.V[i]);
        if (__syncthreads_or(bad) && threadIdx.x == 0) atomicMin(first_bad, o);
    }
}

// ------------------------------------------------------------------ decimation
template <typename VI, int T>
__global__ void __launch_bounds__(T) k_decimate(Meshes M, const int* __restrict__ objs, int n_objs, uint8_t* gstore,
                                                const int64_t* __restrict__ gstore_off, uint32_t* __restrict__ lodF,
                                                int64_t Ftot, uint32_t* __restrict__ lodCnt) {
    constexpr int NW = T / 32;
    extern __shared__ __align__(16) uint8_t dsm[];
    __shared__ double s_len[NW];
    __shared__ uint32_t s_a[NW], s_b[NW], s_red[3][NW], s_third[2];
    __shared__ int s_nsh, s_fuv, s_fvu, s_alive;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = blockIdx.x; i < n_objs; i += gridDim.x) {
        const int o = objs[i];
        const int64_t v0 = M.voff[o], f0 = M.foff[o];
        const uint32_t n = (uint32_t)(M.voff[o + 1] - v0), m = (uint32_t)(M.foff[o + 1] - f0);
        const float* P = M.V + 3 * v0;
        uint8_t* base = gstore ? gstore + gstore_off[i] : dsm;
        VI* fv = reinterpret_cast<VI*>(base);
        uint8_t* fl = base + round16(3 * (size_t)m * sizeof(VI));
        uint32_t* Mu = reinterpret_cast<uint32_t*>(fl + round16(m));
        const uint32_t W = (n + 31) / 32;
        uint32_t *Mv = Mu + W, *M1 = Mu + 2 * W, *M2 = Mu + 3 * W;
        for (uint32_t f = tid; f < m; f += T) {
            for (int k = 0; k < 3; ++k) fv[3 * f + k] = (VI)M.F[3 * (f0 + f) + k];
            fl[f] = 1;  // bit 0 live, bit 1 + j: edge (j, j + 1) refused
        }
        for (uint32_t w = tid; w < 4 * W; w += T) Mu[w] = 0;
        if (tid == 0) s_alive = (int)m;
        __syncthreads();
        // this thread's smallest candidate key and the facet holding it; a full
        // rescan (dirty) is needed only when that facet changes, any other
        // changed facet is folded in
        bool dirty = true;
        double bl = INFINITY;
        uint32_t ba = UINT_MAX, bb = UINT_MAX, bf = UINT_MAX;
        int li = kDecLods - 1;
        while (li >= 0) {
            const uint32_t target = (uint32_t)((uint64_t)m * (uint64_t)(20 * (li + 1)) / 100);  // LOD 20 (li + 1)
            bool snap = (uint32_t)s_alive <= target;
            uint32_t u = 0, v = 0;
            if (!snap) {
                if (dirty) {  // smallest key among this thread's candidate edges
                    bl = INFINITY;
                    ba = bb = bf = UINT_MAX;
                    for (uint32_t f = tid; f < m; f += T) {
                        const uint32_t fla = fl[f];
                        if (fla & 1) fold_facet(P, fv, f, fla, bl, ba, bb, bf);
                    }
                    dirty = false;
                }
                double L = bl;
                uint32_t A = ba, B = bb;
#pragma unroll
                for (int s = 16; s > 0; s >>= 1) {
                    const double L2 = __shfl_xor_sync(0xffffffffu, L, s);
                    const uint32_t A2 = __shfl_xor_sync(0xffffffffu, A, s), B2 = __shfl_xor_sync(0xffffffffu, B, s);
                    if (key_less(L2, A2, B2, L, A, B)) { L = L2; A = A2; B = B2; }
                }
                if (lane == 0) { s_len[wid] = L; s_a[wid] = A; s_b[wid] = B; }
                __syncthreads();
                if (wid == 0) {
                    L = lane < NW ? s_len[lane] : INFINITY;
                    A = lane < NW ? s_a[lane] : UINT_MAX;
                    B = lane < NW ? s_b[lane] : UINT_MAX;
#pragma unroll
                    for (int s = 16; s > 0; s >>= 1) {
                        const double L2 = __shfl_xor_sync(0xffffffffu, L, s);
                        const uint32_t A2 = __shfl_xor_sync(0xffffffffu, A, s), B2 = __shfl_xor_sync(0xffffffffu, B, s);
                        if (key_less(L2, A2, B2, L, A, B)) { L = L2; A = A2; B = B2; }
                    }
                    if (lane == 0) {
                        s_len[0] = L; s_a[0] = A; s_b[0] = B;
                        s_nsh = 0; s_fuv = 0; s_fvu = 0;
                    }
                }
                __syncthreads();
                snap = !(s_len[0] < INFINITY);  // no candidate edge left
                u = s_a[0];
                v = s_b[0];
            }
            if (snap) {  // LOD li: the live facets in index order
                uint32_t pos = 0;
                uint32_t* out = lodF + (size_t)li * 3 * Ftot + 3 * f0;
                for (uint32_t c = 0; c < m; c += T) {
                    const uint32_t f = c + tid;
                    const bool al = f < m && (fl[f] & 1);
                    const unsigned bal = __ballot_sync(0xffffffffu, al);
                    if (lane == 0) s_red[0][wid] = __popc(bal);
                    __syncthreads();
                    uint32_t before = 0, total = 0;
                    for (int w = 0; w < NW; ++w) {
                        const uint32_t x = s_red[0][w];
                        total += x;
                        if (w < wid) before += x;
                    }
                    if (al) {
                        const uint32_t at = pos + before + __popc(bal & ((1u << lane) - 1u));
                        for (int k = 0; k < 3; ++k) out[3 * (size_t)at + k] = fv[3 * f + k];
                    }
                    pos += total;
                    __syncthreads();
                }
                if (tid == 0) lodCnt[(size_t)o * kDecLods + li] = pos;
                --li;
                continue;
            }
            // scan 1: facets around u and v -- shared facets, neighbour masks, normals
            for (uint32_t f = tid; f < m; f += T) {
                if (!(fl[f] & 1)) continue;
                const uint32_t x = fv[3 * f], y = fv[3 * f + 1], z = fv[3 * f + 2];
                const bool hu = x == u || y == u || z == u, hv = x == v || y == v || z == v;
                if (!hu && !hv) continue;
                if (hu && hv) {
                    const int k = atomicAdd(&s_nsh, 1);
                    if (k < 2) s_third[k] = (x != u && x != v) ? x : (y != u && y != v) ? y : z;
                }
                if (hu) mark(Mu, x, y, z, u);
                if (hv) mark(Mv, x, y, z, v);
                if (hu && !hv && turns(P, x, y, z, u, v)) s_fuv = 1;
                if (hv && !hu && turns(P, x, y, z, v, u)) s_fvu = 1;
            }
            __syncthreads();
            const bool cand = s_nsh == 2 && s_third[0] != s_third[1];
            const uint32_t w1 = s_third[0], w2 = s_third[1];
            if (cand) {  // scan 2: neighbours of the two third vertices
                for (uint32_t f = tid; f < m; f += T) {
                    if (!(fl[f] & 1)) continue;
                    const uint32_t x = fv[3 * f], y = fv[3 * f + 1], z = fv[3 * f + 2];
                    if (x == w1 || y == w1 || z == w1) mark(M1, x, y, z, w1);
                    if (x == w2 || y == w2 || z == w2) mark(M2, x, y, z, w2);
                }
                __syncthreads();
            }
            // mask counts (and clear)
            uint32_t c0 = 0, c1 = 0, c2 = 0;
            for (uint32_t w = tid; w < W; w += T) {
                c0 += __popc(Mu[w] & Mv[w]);
                c1 += __popc(M1[w]);
                c2 += __popc(M2[w]);
                Mu[w] = Mv[w] = M1[w] = M2[w] = 0;
            }
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                c0 += __shfl_xor_sync(0xffffffffu, c0, s);
                c1 += __shfl_xor_sync(0xffffffffu, c1, s);
                c2 += __shfl_xor_sync(0xffffffffu, c2, s);
            }
            if (lane == 0) { s_red[0][wid] = c0; s_red[1][wid] = c1; s_red[2][wid] = c2; }
            __syncthreads();
            c0 = c1 = c2 = 0;
            for (int w = 0; w < NW; ++w) { c0 += s_red[0][w]; c1 += s_red[1][w]; c2 += s_red[2][w]; }
            const bool link = cand && c0 == 2 && c1 > 3 && c2 > 3;
            int mode = 0;  // 0: refuse the edge, 1: collapse r into k
            uint32_t r = 0, k = 0;
            if (link && !s_fuv) { mode = 1; r = u; k = v; }
            else if (link && !s_fvu) { mode = 1; r = v; k = u; }
            // scan 3: apply
            int kills = 0;
            for (uint32_t f = tid; f < m; f += T) {
                const uint32_t fla = fl[f];
                if (!(fla & 1)) continue;
                VI* t = fv + 3 * f;
                const uint32_t x = t[0], y = t[1], z = t[2];
                if (mode) {
                    const bool hr = x == r || y == r || z == r, hk = x == k || y == k || z == k;
                    if (hr && hk) { fl[f] = 0; ++kills; dirty |= f == bf; continue; }
                    if (!hr && !hk) continue;
                    if (hr) {
                        if (x == r) t[0] = (VI)k;
                        if (y == r) t[1] = (VI)k;
                        if (z == r) t[2] = (VI)k;
                    }
                    uint32_t nf = fla;  // every edge at k is a candidate again
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        if ((uint32_t)t[j] == k || (uint32_t)t[j == 2 ? 0 : j + 1] == k) nf &= ~(2u << j);
                    fl[f] = (uint8_t)nf;
                    if (f == bf) dirty = true;  // its old keys may have been the minimum
                    else fold_facet(P, fv, f, nf, bl, ba, bb, bf);
                } else {
                    const bool hu = x == u || y == u || z == u, hv = x == v || y == v || z == v;
                    if (!(hu && hv)) continue;
                    uint32_t nf = fla;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const uint32_t a = t[j], b = t[j == 2 ? 0 : j + 1];
                        if ((a == u && b == v) || (a == v && b == u)) nf |= 2u << j;
                    }
                    fl[f] = (uint8_t)nf;
                    dirty |= f == bf;  // slots only left the candidates
                }
            }
            if (kills) atomicSub(&s_alive, kills);
            __syncthreads();
        }
        __syncthreads();  // the next object reuses the storage
    }
}

// ------------------------------------------------------------------ block helpers
template <int T>
__device__ __forceinline__ uint32_t block_count_before(bool flag, uint32_t* red, uint32_t& total) {
    constexpr int NW = T / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) red[wid] = __popc(bal);
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (int w = 0; w < NW; ++w) {
        const uint32_t x = red[w];
        total += x;
        if (w < wid) before += x;
    }
    __syncthreads();
    return before + __popc(bal & ((1u << lane) - 1u));
}

// exclusive scan of x over the block's threads (in thread order)
template <int T>
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t x, uint32_t* red, uint32_t& total) {
    constexpr int NW = T / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, s);
        if (lane >= s) incl += y;
    }
    if (lane == 31) red[wid] = incl;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (int w = 0; w < NW; ++w) {
        const uint32_t y = red[w];
        total += y;
        if (w < wid) before += y;
    }
    __syncthreads();
    return before + incl - x;
}

// nearest of the points c[0..k) (double triples) to p; ties to the lowest index
__device__ __forceinline__ uint32_t nearest(double3 p, const double* c, uint32_t k, double& best) {
    uint32_t g = 0;
    best = INFINITY;
    for (uint32_t s = 0; s < k; ++s) {
        const double d = dist2(p, make_double3(c[3 * s], c[3 * s + 1], c[3 * s + 2]));
        if (d < best) { best = d; g = s; }
    }
    return g;
}

// nearest core (vertex ids) to p; ties to the lowest voxel
__device__ __forceinline__ uint32_t nearest_core(double3 p, const float* P, const uint32_t* core, uint32_t k) {
    uint32_t g = 0;
    double best = INFINITY;
    for (uint32_t s = 0; s < k; ++s) {
        const double d = dist2(p, vtx(P, core[s]));
        if (d < best) { best = d; g = s; }
    }
    return g;
}

// ------------------------------------------------------------------ voxels
template <int T>
__global__ void __launch_bounds__(T) k_voxels(Meshes M, int voxel_size, const uint32_t* __restrict__ lodF,
                                              const uint32_t* __restrict__ lodCnt, VoxScratch S,
                                              unsigned long long* __restrict__ obj_bytes) {
    constexpr int NW = T / 32;
    __shared__ double s_v[NW];
    __shared__ uint32_t s_i[NW], s_red[NW];
    __shared__ uint32_t s_cur, s_nvox;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int o = blockIdx.x; o < M.n; o += gridDim.x) {
        const int64_t v0 = M.voff[o], f0 = M.foff[o], s0 = S.soff[o];
        const uint32_t n = (uint32_t)(M.voff[o + 1] - v0), m = (uint32_t)(M.foff[o + 1] - f0);
        const uint32_t ns = m / (uint32_t)voxel_size + 1;
        const float* P = M.V + 3 * v0;
        const uint32_t* F100 = M.F + 3 * f0;
        double* sd = S.seed + 3 * s0;
        double* dmin = S.dmin + v0;
        uint32_t* asg = S.asg + v0;
        // 2a. farthest-point seeds from vertex 0
        uint32_t cur = 0;
        for (uint32_t s = 0; s < ns; ++s) {
            const double3 c = vtx(P, cur);
            if (tid == 0) { sd[3 * s] = c.x; sd[3 * s + 1] = c.y; sd[3 * s + 2] = c.z; }
            double bv = -1.0;
            uint32_t bi = UINT_MAX;
            for (uint32_t i = tid; i < n; i += T) {
                const double d = sqrt(dist2(vtx(P, i), c));
                const double dm = s == 0 ? d : fmin(dmin[i], d);
                dmin[i] = dm;
                if (dm > bv) { bv = dm; bi = i; }
            }
#pragma unroll
            for (int k = 16; k > 0; k >>= 1) {
                const double v2 = __shfl_xor_sync(0xffffffffu, bv, k);
                const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, k);
                if (v2 > bv || (v2 == bv && i2 < bi)) { bv = v2; bi = i2; }
            }
            if (lane == 0) { s_v[wid] = bv; s_i[wid] = bi; }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < NW; ++w)
                    if (s_v[w] > bv || (s_v[w] == bv && s_i[w] < bi)) { bv = s_v[w]; bi = s_i[w]; }
                s_cur = bi;
            }
            __syncthreads();
            cur = s_cur;
        }
        // 2b. two Lloyd steps
        for (int it = 0; it < 2; ++it) {
            for (uint32_t i = tid; i < n; i += T) {
                double d;
                asg[i] = nearest(vtx(P, i), sd, ns, d);
            }
            __syncthreads();
            for (uint32_t s = tid; s < ns; s += T) {  // sums in vertex order
                double ax = 0.0, ay = 0.0, az = 0.0;
                uint32_t cnt = 0;
                for (uint32_t i = 0; i < n; ++i)
                    if (asg[i] == s) {
                        const double3 p = vtx(P, i);
                        ax = ax + p.x; ay = ay + p.y; az = az + p.z;
                        ++cnt;
                    }
                if (cnt) {
                    const double r = 1.0 / (double)cnt;
                    sd[3 * s] = ax * r; sd[3 * s + 1] = ay * r; sd[3 * s + 2] = az * r;
                }
            }
            __syncthreads();
        }
        // 2c. facets to seeds by barycentre; a seed's nearest facet gives its core
        unsigned long long* bestd = S.bestd + s0;
        uint32_t* bestf = S.bestf + s0;
        for (uint32_t s = tid; s < ns; s += T) { bestd[s] = ~0ull; bestf[s] = UINT_MAX; }
        __syncthreads();
        for (int pass = 0; pass < 2; ++pass) {
            for (uint32_t f = tid; f < m; f += T) {
                const double3 a = vtx(P, F100[3 * f]), b = vtx(P, F100[3 * f + 1]), c = vtx(P, F100[3 * f + 2]);
                const double k3 = 1.0 / 3.0;
                const double3 q = make_double3(((a.x + b.x) + c.x) * k3, ((a.y + b.y) + c.y) * k3, ((a.z + b.z) + c.z) * k3);
                double d;
                const uint32_t g = nearest(q, sd, ns, d);
                const unsigned long long bits = (unsigned long long)__double_as_longlong(d);
                if (pass == 0) atomicMin(bestd + g, bits);
                else if (bestd[g] == bits) atomicMin(bestf + g, f);
            }
            __syncthreads();
        }
        uint32_t* core = S.core + s0;
        uint32_t nvox = 0;
        for (uint32_t c0 = 0; c0 < ns; c0 += T) {  // cores of the seeds with a facet, in seed order
            const uint32_t s = c0 + tid;
            const bool has = s < ns && bestf[s] != UINT_MAX;
            const uint32_t fb = has ? bestf[s] : 0;
            uint32_t total;
            const uint32_t at = block_count_before<T>(has, s_red, total);
            if (has) core[nvox + at] = F100[3 * fb];
            nvox += total;
        }
        __syncthreads();
        // 3. LOD-100 triangles to cores; keep the cores that receive one
        uint32_t* cnt100 = S.vcnt + (size_t)(kNumLods - 1) * S.Stot + s0;
        for (uint32_t v = tid; v < nvox; v += T) cnt100[v] = 0;
        __syncthreads();
        for (uint32_t f = tid; f < m; f += T) atomicAdd(cnt100 + nearest_core(vtx(P, F100[3 * f]), P, core, nvox), 1u);
        __syncthreads();
        uint32_t kept = 0;
        for (uint32_t c0 = 0; c0 < nvox; c0 += T) {  // in place: kept cores move down
            const uint32_t v = c0 + tid;
            const bool has = v < nvox && cnt100[v] > 0;
            const uint32_t cv = has ? core[v] : 0;
            uint32_t total;
            const uint32_t at = block_count_before<T>(has, s_red, total);
            if (has) core[kept + at] = cv;
            kept += total;
            __syncthreads();
        }
        nvox = kept;
        // every LOD: triangles to the kept voxels, grouped by voxel in LOD order
        uint32_t ntri = 0;
        for (int l = 0; l < kNumLods; ++l) {
            const uint32_t* LF = l < kNumLods - 1 ? lodF + (size_t)l * 3 * S.Ftot + 3 * f0 : F100;
            const uint32_t cl = l < kNumLods - 1 ? lodCnt[(size_t)o * kDecLods + l] : m;
            uint32_t* tv = S.tvox + (size_t)l * S.Ftot + f0;
            uint32_t* od = S.ord + (size_t)l * S.Ftot + f0;
            uint32_t* vc = S.vcnt + (size_t)l * S.Stot + s0;
            uint32_t* vs = S.vst + (size_t)l * S.Stot + s0;
            for (uint32_t v = tid; v < nvox; v += T) vc[v] = 0;
            __syncthreads();
            for (uint32_t t = tid; t < cl; t += T) {
                const uint32_t g = nearest_core(vtx(P, LF[3 * t]), P, core, nvox);
                tv[t] = g;
                atomicAdd(vc + g, 1u);
            }
            __syncthreads();
            uint32_t run = 0;
            for (uint32_t c0 = 0; c0 < nvox; c0 += T) {
                const uint32_t v = c0 + tid;
                const uint32_t x = v < nvox ? vc[v] : 0;
                uint32_t total;
                const uint32_t at = block_excl_sum<T>(x, s_red, total);
                if (v < nvox) vs[v] = run + at;
                run += total;
            }
            __syncthreads();
            for (uint32_t v = tid; v < nvox; v += T) {  // stable: each voxel walks the LOD in order
                uint32_t c = vs[v];
                for (uint32_t t = 0; t < cl; ++t)
                    if (tv[t] == v) od[c++] = t;
            }
            ntri += cl;
            __syncthreads();
        }
        if (tid == 0) {
            S.nvox[o] = nvox;
            obj_bytes[o] = 68ull + 44ull * ntri + 116ull * nvox;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ RAW writer
// Object o's bytes start at word pos[o] / 4 of `out` (every object is a
// multiple of 4 bytes long and the batch starts on an object).
template <int T>
__global__ void __launch_bounds__(T) k_write(Meshes M, const uint32_t* __restrict__ lodF, const uint32_t* __restrict__ lodCnt,
                                             VoxScratch S, const unsigned long long* __restrict__ pos,
                                             uint32_t* __restrict__ out) {
    constexpr int NW = T / 32;
    __shared__ float s_f[6][NW];
    __shared__ float s_d[NW];
    __shared__ uint32_t s_i[NW];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int o = blockIdx.x; o < M.n; o += gridDim.x) {
        const int64_t v0 = M.voff[o], f0 = M.foff[o], s0 = S.soff[o];
        const uint32_t n = (uint32_t)(M.voff[o + 1] - v0), m = (uint32_t)(M.foff[o + 1] - f0);
        const float* P = M.V + 3 * v0;
        const uint32_t nvox = S.nvox[o];
        const uint32_t* core = S.core + s0;
        uint32_t* W = out + pos[o] / 4;
        uint32_t cl[kNumLods], lstart[kNumLods], ntri = 0;
        for (int l = 0; l < kNumLods; ++l) {
            cl[l] = l < kNumLods - 1 ? lodCnt[(size_t)o * kDecLods + l] : m;
            lstart[l] = ntri;
            ntri += cl[l];
        }
        const uint64_t data = 44ull * ntri;
        if (tid == 0) { W[0] = (uint32_t)data; W[1] = (uint32_t)(data >> 32); }
        uint32_t* D = W + 2;
        for (int l = 0; l < kNumLods; ++l) {
            const uint32_t* LF = l < kNumLods - 1 ? lodF + (size_t)l * 3 * S.Ftot + 3 * f0 : M.F + 3 * f0;
            const uint32_t* tv = S.tvox + (size_t)l * S.Ftot + f0;
            const uint32_t* od = S.ord + (size_t)l * S.Ftot + f0;
            const uint32_t* vc = S.vcnt + (size_t)l * S.Stot + s0;
            const uint32_t* vs = S.vst + (size_t)l * S.Stot + s0;
            for (uint32_t g = tid; g < cl[l]; g += T) {
                const uint32_t t = od[g], v = tv[t], sv = vs[v], cv = vc[v], j = g - sv;
                uint32_t* grp = D + 11 * (size_t)(lstart[l] + sv);
                uint32_t* c = grp + 9 * j;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float* q = P + 3 * (size_t)LF[3 * t + k];
                    c[3 * k] = __float_as_uint(q[0]);
                    c[3 * k + 1] = __float_as_uint(q[1]);
                    c[3 * k + 2] = __float_as_uint(q[2]);
                }
                grp[9 * cv + 2 * j] = 0u;
                grp[9 * cv + 2 * j + 1] = 0u;
            }
        }
        uint32_t* H = D + 11 * (size_t)ntri;
        if (tid == 0) { H[0] = nvox; H[1] = 0u; }
        if (tid < 2 * kNumLods) H[2 + tid] = 0u;  // object-level bounds
        for (uint32_t v = tid; v < nvox; v += T) {
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int l = 0; l < kNumLods; ++l) {
                const uint32_t* LF = l < kNumLods - 1 ? lodF + (size_t)l * 3 * S.Ftot + 3 * f0 : M.F + 3 * f0;
                const uint32_t* od = S.ord + (size_t)l * S.Ftot + f0;
                const uint32_t sv = S.vst[(size_t)l * S.Stot + s0 + v], cv = S.vcnt[(size_t)l * S.Stot + s0 + v];
                for (uint32_t g = sv; g < sv + cv; ++g)
                    for (int k = 0; k < 3; ++k) {
                        const float* q = P + 3 * (size_t)LF[3 * od[g] + k];
                        for (int d = 0; d < 3; ++d) {  // a tie keeps the value held (-0 vs +0)
                            lo[d] = q[d] < lo[d] ? q[d] : lo[d];
                            hi[d] = hi[d] < q[d] ? q[d] : hi[d];
                        }
                    }
            }
            uint32_t* R = H + 12 + 29 * (size_t)v;
            for (int d = 0; d < 3; ++d) { R[d] = __float_as_uint(lo[d]); R[3 + d] = __float_as_uint(hi[d]); }
            for (int d = 0; d < 3; ++d) R[6 + d] = __float_as_uint(P[3 * (size_t)core[v] + d]);
            for (int l = 0; l < kNumLods; ++l) {
                const uint64_t off = 44ull * (lstart[l] + S.vst[(size_t)l * S.Stot + s0 + v]);
                const uint32_t cv = S.vcnt[(size_t)l * S.Stot + s0 + v];
                R[9 + 4 * l] = (uint32_t)off;
                R[10 + 4 * l] = (uint32_t)(off >> 32);
                R[11 + 4 * l] = cv;
                R[12 + 4 * l] = 0u;
            }
        }
        // 4. transform: the vertex nearest the centre of the float bounding box
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = tid; i < n; i += T)
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], P[3 * (size_t)i + d]);
                hi[d] = fmaxf(hi[d], P[3 * (size_t)i + d]);
            }
#pragma unroll
        for (int k = 16; k > 0; k >>= 1)
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], k));
                hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], k));
            }
        if (lane == 0)
            for (int d = 0; d < 3; ++d) { s_f[d][wid] = lo[d]; s_f[3 + d][wid] = hi[d]; }
        __syncthreads();
        for (int w = 0; w < NW; ++w)
            for (int d = 0; d < 3; ++d) { lo[d] = fminf(lo[d], s_f[d][w]); hi[d] = fmaxf(hi[d], s_f[3 + d][w]); }
        const float cx = 0.5f * (lo[0] + hi[0]), cy = 0.5f * (lo[1] + hi[1]), cz = 0.5f * (lo[2] + hi[2]);
        float bd = INFINITY;
        uint32_t bi = UINT_MAX;
        for (uint32_t i = tid; i < n; i += T) {
            const float dx = P[3 * (size_t)i] - cx, dy = P[3 * (size_t)i + 1] - cy, dz = P[3 * (size_t)i + 2] - cz;
            const float d = dx * dx + dy * dy + dz * dz;
            if (d < bd) { bd = d; bi = i; }
        }
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) {
            const float d2 = __shfl_xor_sync(0xffffffffu, bd, k);
            const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, k);
            if (d2 < bd || (d2 == bd && i2 < bi)) { bd = d2; bi = i2; }
        }
        if (lane == 0) { s_d[wid] = bd; s_i[wid] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < NW; ++w)
                if (s_d[w] < bd || (s_d[w] == bd && s_i[w] < bi)) { bd = s_d[w]; bi = s_i[w]; }
            uint32_t* X = H + 12 + 29 * (size_t)nvox;
            for (int d = 0; d < 3; ++d) X[d] = __float_as_uint(P[3 * (size_t)bi + d]);
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace tdp

// ------------------------------------------------------------------ host driver
using namespace tdp;

namespace {

struct DevMem {  // allocations of one batch, back to the context's block cache on every return
    tdp_ctx* ctx;
    std::vector<void*> ps;
    ~DevMem() {
        cudaStreamSynchronize(ctx->stream);  // nothing queued may still use a block
        for (void* p : ps) block_release(ctx, p);
    }
    template <typename X>
    cudaError_t get(X** p, size_t count) {
        void* q = nullptr;
        const cudaError_t e = block_alloc(ctx, &q, std::max<size_t>(count, 1) * sizeof(X));
        if (e == cudaSuccess) ps.push_back(q);
        *p = (X*)q;
        return e;
    }
};

inline size_t upper_bytes(int64_t m, int voxel_size) {  // RAW bytes of an object, at most
    return 68 + 44 * (size_t)kNumLods * (size_t)m + 116 * ((size_t)m / (size_t)voxel_size + 1);
}

}  // namespace

extern "C" int tdp_raw_prep_bound(const int64_t* face_off, long n_objects, int voxel_size, size_t* max_len) {
    if (!max_len || n_objects < 0 || voxel_size <= 0 || (n_objects > 0 && !face_off)) return TDP_ERR_ARG;
    size_t s = 1;
    for (long o = 0; o < n_objects; ++o) {
        const int64_t m = face_off[o + 1] - face_off[o];
        if (m < 0) return TDP_ERR_ARG;
        s += upper_bytes(m, voxel_size);
    }
    *max_len = s;
    return TDP_OK;
}

extern "C" int tdp_raw_from_meshes(tdp_ctx* ctx, const float* vertices, const int64_t* vert_off, const uint32_t* faces,
                                   const int64_t* face_off, long n_objects, int voxel_size, void* out, size_t cap,
                                   size_t* len, tdp_prep_info* info) {
    if (!ctx) return TDP_ERR_ARG;
    if (n_objects < 0 || n_objects > INT_MAX || voxel_size <= 0 || (n_objects > 0 && (!vertices || !vert_off || !faces || !face_off)))
        return fail(ctx, TDP_ERR_ARG, "tdp_raw_from_meshes: bad arguments");
    for (long o = 0; o < n_objects; ++o)
        if (vert_off[o + 1] < vert_off[o] || face_off[o + 1] < face_off[o] || vert_off[o] < 0 || face_off[o] < 0)
            return fail(ctx, TDP_ERR_ARG, "tdp_raw_from_meshes: offsets must be non-decreasing");
    const auto t_start = std::chrono::steady_clock::now();
    tdp_prep_info inf{};
    inf.n_objects = n_objects;
    cudaStream_t s = ctx->stream;
#define CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string("tdp_raw_from_meshes: " #x ": ") + cudaGetErrorString(_e)); } while (0)
    // batches of consecutive objects within a device-memory budget
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    // a batch holds at most min(6 GiB, a quarter of the free memory, an eighth of the context's cap)
    size_t budget = std::min<size_t>((size_t)6 << 30, free_b / 4);
    if (ctx->budget) budget = std::min(budget, ctx->budget / 8);
    budget = std::max<size_t>(budget, (size_t)16 << 20);
    std::vector<long> cuts{0};
    {
        size_t acc = 0;
        for (long o = 0; o < n_objects; ++o) {
            const int64_t n = vert_off[o + 1] - vert_off[o], m = face_off[o + 1] - face_off[o];
            const size_t need = 24 * (size_t)n + (12 + 48 + 40) * (size_t)m + 80 * ((size_t)m / voxel_size + 1) +
                                upper_bytes(m, voxel_size) + dec_bytes(n, m, 4) + 64;
            if (acc > 0 && acc + need > budget) {
                cuts.push_back(o);
                acc = 0;
            }
            acc += need;
        }
        cuts.push_back(n_objects);
    }
    size_t pos_out = 1;  // the tile's type byte
    std::vector<unsigned long long> bytes;
    cudaEvent_t ev[4];
    for (auto& e : ev) CU(cudaEventCreate(&e));
    struct EvFree {
        cudaEvent_t* e;
        ~EvFree() { for (int k = 0; k < 4; ++k) cudaEventDestroy(e[k]); }
    } evfree{ev};
    for (size_t b = 0; b + 1 < cuts.size(); ++b) {
        const long o0 = cuts[b], o1 = cuts[b + 1], nb = o1 - o0;
        if (nb <= 0) continue;
        DevMem dm{ctx, {}};
        const int64_t vb = vert_off[o0], fb = face_off[o0];
        const int64_t Vtot = vert_off[o1] - vb, Ftot = face_off[o1] - fb;
        std::vector<int64_t> voff(nb + 1), foff(nb + 1), soff(nb + 1);
        soff[0] = 0;
        for (long i = 0; i <= nb; ++i) {
            voff[i] = vert_off[o0 + i] - vb;
            foff[i] = face_off[o0 + i] - fb;
            if (i < nb) soff[i + 1] = soff[i] + (face_off[o0 + i + 1] - face_off[o0 + i]) / voxel_size + 1;
        }
        const int64_t Stot = soff[nb];
        float* dV;
        uint32_t* dF;
        int64_t *dvoff, *dfoff, *dsoff;
        int* dbad;
        CU(dm.get(&dV, 3 * (size_t)Vtot));
        CU(dm.get(&dF, 3 * (size_t)Ftot));
        CU(dm.get(&dvoff, nb + 1));
        CU(dm.get(&dfoff, nb + 1));
        CU(dm.get(&dsoff, nb + 1));
        CU(dm.get(&dbad, 1));
        CU(cudaMemcpyAsync(dV, vertices + 3 * vb, 12 * (size_t)Vtot, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dF, faces + 3 * fb, 12 * (size_t)Ftot, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dvoff, voff.data(), 8 * (nb + 1), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dfoff, foff.data(), 8 * (nb + 1), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dsoff, soff.data(), 8 * (nb + 1), cudaMemcpyHostToDevice, s));
        const int big = INT_MAX;
        CU(cudaMemcpyAsync(dbad, &big, 4, cudaMemcpyHostToDevice, s));
        Meshes Mh{dV, dvoff, dF, dfoff, (int)nb};
        k_validate<<<(int)std::min<long>(nb, 65535), 256, 0, s>>>(Mh, dbad);
        CU(cudaGetLastError());
        int bad = INT_MAX;
        CU(cudaMemcpyAsync(&bad, dbad, 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (bad != INT_MAX)
            return fail(ctx, TDP_ERR_ARG, "tdp_raw_from_meshes: object " + std::to_string(o0 + bad) +
                                              " has no vertex or facet, a vertex index out of range, a facet repeating "
                                              "a vertex or a non-finite coordinate");
        CU(cudaEventRecord(ev[0], s));
        // 1. decimation, three launch shapes by the object's storage
        uint32_t *lodF, *lodCnt;
        CU(dm.get(&lodF, (size_t)kDecLods * 3 * Ftot));
        CU(dm.get(&lodCnt, (size_t)kDecLods * nb));
        std::vector<int> small, large, huge;
        std::vector<int64_t> hoff{0};
        size_t s_small = 0, s_large = 0;
        for (long i = 0; i < nb; ++i) {
            const int64_t n = voff[i + 1] - voff[i], m = foff[i + 1] - foff[i];
            const size_t b16 = dec_bytes(n, m, 2);
            if (n <= 65535 && b16 <= kSmemSmall) { small.push_back((int)i); s_small = std::max(s_small, b16); }
            else if (n <= 65535 && b16 <= kSmemLarge) { large.push_back((int)i); s_large = std::max(s_large, b16); }
            else { huge.push_back((int)i); hoff.push_back(hoff.back() + (int64_t)dec_bytes(n, m, 4)); }
        }
        int* dl;
        CU(dm.get(&dl, small.size() + large.size() + huge.size()));
        std::vector<int> all(small);
        all.insert(all.end(), large.begin(), large.end());
        all.insert(all.end(), huge.begin(), huge.end());
        if (!all.empty()) CU(cudaMemcpyAsync(dl, all.data(), 4 * all.size(), cudaMemcpyHostToDevice, s));
        if (!small.empty()) {
            auto kern = k_decimate<uint16_t, 128>;
            CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_small));
            kern<<<(int)std::min<size_t>(small.size(), 1u << 30), 128, s_small, s>>>(Mh, dl, (int)small.size(), nullptr,
                                                                                    nullptr, lodF, Ftot, lodCnt);
            CU(cudaGetLastError());
        }
        if (!large.empty()) {
            auto kern = k_decimate<uint16_t, 1024>;
            CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_large));
            kern<<<(int)large.size(), 1024, s_large, s>>>(Mh, dl + small.size(), (int)large.size(), nullptr, nullptr,
                                                         lodF, Ftot, lodCnt);
            CU(cudaGetLastError());
        }
        if (!huge.empty()) {
            uint8_t* gst;
            int64_t* dho;
            CU(dm.get(&gst, (size_t)hoff.back()));
            CU(dm.get(&dho, hoff.size()));
            CU(cudaMemcpyAsync(dho, hoff.data(), 8 * hoff.size(), cudaMemcpyHostToDevice, s));
            k_decimate<uint32_t, 1024><<<(int)huge.size(), 1024, 0, s>>>(Mh, dl + small.size() + large.size(),
                                                                      (int)huge.size(), gst, dho, lodF, Ftot, lodCnt);
            CU(cudaGetLastError());
        }
        CU(cudaEventRecord(ev[1], s));
        // 2-3. voxels
        VoxScratch S{};
        CU(dm.get(&S.dmin, (size_t)Vtot));
        CU(dm.get(&S.asg, (size_t)Vtot));
        CU(dm.get(&S.seed, 3 * (size_t)Stot));
        CU(dm.get(&S.bestd, (size_t)Stot));
        CU(dm.get(&S.bestf, (size_t)Stot));
        CU(dm.get(&S.core, (size_t)Stot));
        CU(dm.get(&S.nvox, (size_t)nb));
        CU(dm.get(&S.tvox, (size_t)kNumLods * Ftot));
        CU(dm.get(&S.ord, (size_t)kNumLods * Ftot));
        CU(dm.get(&S.vcnt, (size_t)kNumLods * Stot));
        CU(dm.get(&S.vst, (size_t)kNumLods * Stot));
        S.soff = dsoff;
        S.Ftot = Ftot;
        S.Stot = Stot;
        unsigned long long *dbytes, *dpos;
        CU(dm.get(&dbytes, (size_t)nb));
        CU(dm.get(&dpos, (size_t)nb));
        k_voxels<kPrepThreads><<<(int)nb, kPrepThreads, 0, s>>>(Mh, voxel_size, lodF, lodCnt, S, dbytes);
        CU(cudaGetLastError());
        CU(cudaEventRecord(ev[2], s));
        bytes.assign(nb, 0);
        float ms_vox[2] = {0, 0};
        std::vector<uint32_t> hcnt((size_t)kDecLods * nb), hnvox(nb);
        CU(cudaMemcpyAsync(bytes.data(), dbytes, 8 * nb, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(hcnt.data(), lodCnt, 4 * hcnt.size(), cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(hnvox.data(), S.nvox, 4 * nb, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms_vox[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms_vox[1], ev[1], ev[2]);
        inf.decimate_ms += ms_vox[0];
        inf.voxel_ms += ms_vox[1];
        std::vector<unsigned long long> hpos(nb);
        unsigned long long run = 0;
        for (long i = 0; i < nb; ++i) {
            hpos[i] = run;
            run += bytes[i];
            for (int l = 0; l < kDecLods; ++l) inf.n_triangles[l] += hcnt[(size_t)i * kDecLods + l];
            inf.n_triangles[kNumLods - 1] += foff[i + 1] - foff[i];
            inf.n_voxels += hnvox[i];
        }
        // 4. RAW bytes of the batch, then to the caller's buffer
        if (out && pos_out + run <= cap) {
            uint32_t* dout;
            CU(dm.get(&dout, (size_t)(run / 4)));
            CU(cudaMemcpyAsync(dpos, hpos.data(), 8 * nb, cudaMemcpyHostToDevice, s));
            CU(cudaEventRecord(ev[2], s));  // the writer alone (the host's allocation above is not timed)
            k_write<kPrepThreads><<<(int)nb, kPrepThreads, 0, s>>>(Mh, lodF, lodCnt, S, dpos, dout);
            CU(cudaGetLastError());
            CU(cudaEventRecord(ev[3], s));
            CU(cudaMemcpyAsync((uint8_t*)out + pos_out, dout, (size_t)run, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[2], ev[3]);
            inf.write_ms += ms;
        }
        pos_out += (size_t)run;
        inf.batches += 1;
    }
#undef CU
    if (len) *len = pos_out;
    if (!out) {
        if (info) *info = inf;
        return TDP_OK;
    }
    if (cap < pos_out) return fail(ctx, TDP_ERR_ARG, "tdp_raw_from_meshes: output buffer too small");
    ((uint8_t*)out)[0] = kRawType;
    // per-triangle and object-level bounds, on the device
    const auto t_b = std::chrono::steady_clock::now();
    tdp_bounds_info bi{};
    int rc = TDP_OK;
    if (n_objects > 0 && (rc = tdp_raw_compute_bounds(ctx, out, pos_out, out, &bi)) != TDP_OK) return rc;
    const auto t_end = std::chrono::steady_clock::now();
    inf.bounds_ms = std::chrono::duration<double, std::milli>(t_end - t_b).count();
    inf.total_ms = std::chrono::duration<double, std::milli>(t_end - t_start).count();
    if (info) *info = inf;
    return TDP_OK;
}
