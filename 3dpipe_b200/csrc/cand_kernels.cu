// cand_kernels.cu -- object candidates on the GPU.
//
// Restates, for a whole tile of queries at once, what the reference's octree
// returns per query (OctreeNode::query_knn_fast / query_within, reference
// src/index/octree.cpp:120-154, :215-330) -- the same set and the same order
// as the host implementation in src/index/candidates.cpp, which the tests pin
// against the reference octree compiled from source:
//   kNN:    the K objects with the smallest transform distance (ties by id)
//           plus every object whose box gap is below the K-th distance,
//           ordered by (transform distance, id);
//   within: every object with box gap <= tau, ordered by id.
// Both distances use the reference's float operations with no FMA
// contraction (__fmul_rn / __fadd_rn / __fsqrt_rn), so membership at a
// boundary is decided exactly as on the host.
//
// Per query, one warp:
//   k_cand_kth   ring search over a grid of transform points; after each ring
//                the K-th smallest (distance, id) key of the points seen so far
//                is found by bisection, and the search stops once it is inside
//                the ring's radius by more than the grid's rounding slack;
//   k_cand_pass  scans the box-grid cells that the query box, grown by tau or
//                by the K-th distance, overlaps; an object spanning several
//                cells is counted only in its first cell inside the scan
//                range; a count pass sizes the CSR, a write pass emits keys;
// then a CUB segmented sort orders each query's keys.
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include <float.h>

#include <algorithm>
#include <climits>
#include <string>
#include <vector>

#include "cand_kernels.cuh"
#include "index/candidates.h"

namespace tdp {
namespace {

struct DG {
    float lo0, lo1, lo2, cell, slack;
    int n0, n1, n2;
    const int64_t* start;
    const int32_t* items;
};

DG dg(const DevGrid& g) {
    return DG{g.lo[0], g.lo[1], g.lo[2], g.cell, g.slack, g.n[0], g.n[1], g.n[2], g.start, g.items};
}

// (long)floor((v - lo) / cell) clamped to [0, n-1], as CellGrid::ci
__device__ __forceinline__ int dci(float v, float lo, float cell, int n) {
    const float c = floorf(__fdiv_rn(__fsub_rn(v, lo), cell));
    if (!(c > 0.f)) return 0;
    if (c >= (float)(n - 1)) return n - 1;
    return (int)c;
}

__device__ __forceinline__ float d_box_gap(const float* a, const float* b) {
    float m = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float t1 = __fsub_rn(a[i], b[3 + i]);
        const float t2 = __fsub_rn(a[3 + i], b[i]);
        if (t2 < 0.f) m = __fadd_rn(m, __fmul_rn(t2, t2));
        else if (t1 > 0.f) m = __fadd_rn(m, __fmul_rn(t1, t1));
    }
    return __fsqrt_rn(m);
}

__device__ __forceinline__ float d_point_dist(const float* a, const float* b) {
    const float dx = __fsub_rn(a[0], b[0]), dy = __fsub_rn(a[1], b[1]), dz = __fsub_rn(a[2], b[2]);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

// aab::intersect of the reference: the boxes overlap strictly on every axis
__device__ __forceinline__ bool strict_overlap(const float* b, const float* a) {
    return !(b[0] >= a[3] || b[3] <= a[0] || b[1] >= a[4] || b[4] <= a[1] || b[2] >= a[5] || b[5] <= a[2]);
}

__device__ __forceinline__ unsigned long long key_of(float d, int id) {
    return ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)id;
}

constexpr int kWarps = 4;
constexpr int kCap = 1024;  // transform points a warp keeps during one ring search

// smallest key T with count(key <= T) >= K among n keys (n >= K), by bisection
__device__ unsigned long long kth_key(const unsigned long long* keys, int n, int K, int lane) {
    unsigned long long lo = 0, hi = ~0ull;
    while (lo < hi) {
        const unsigned long long mid = lo + (hi - lo) / 2;
        int c = 0;
        for (int i = lane; i < n; i += 32) c += keys[i] <= mid;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (c >= K) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Ring search of one query (one warp): the K-th smallest (transform
// distance, id) key, ~0 when tile 2 holds fewer than K candidates.  The keys
// of the points seen so far go to keys[0, cap); returns false when a ring
// brought more than cap points (the result is then unusable).  Every point of
// tile 2 lies in exactly one grid cell and every cell is visited by exactly
// one ring, so cap >= n2 can never overflow.
__device__ bool kth_search(const DG& pg, const float* xq, const float* __restrict__ xf2, int q, int K, int self,
                           unsigned long long* keys, int cap, int* cnt, int lane, unsigned long long& result) {
    const int cx = dci(xq[0], pg.lo0, pg.cell, pg.n0), cy = dci(xq[1], pg.lo1, pg.cell, pg.n1);
    const int cz = dci(xq[2], pg.lo2, pg.cell, pg.n2);
    if (lane == 0) *cnt = 0;
    __syncwarp();
    const int maxr = max(pg.n0, max(pg.n1, pg.n2));
    result = ~0ull;  // fewer than K objects: every object is a candidate
    bool over = false;
    for (int r = 0; r <= maxr; ++r) {
        const int side = 2 * r + 1;
        const int total = side * side * side;
        for (int t = lane; t < total; t += 32) {
            const int dx = t % side - r, dy = (t / side) % side - r, dz = t / (side * side) - r;
            if (max(abs(dx), max(abs(dy), abs(dz))) != r) continue;
            const int x = cx + dx, y = cy + dy, z = cz + dz;
            if (x < 0 || y < 0 || z < 0 || x >= pg.n0 || y >= pg.n1 || z >= pg.n2) continue;
            const size_t c = ((size_t)x * pg.n1 + y) * pg.n2 + z;
            for (int64_t k = pg.start[c]; k < pg.start[c + 1]; ++k) {
                const int o = pg.items[k];
                if (self && o == q) continue;
                const int pos = atomicAdd(cnt, 1);
                if (pos < cap) keys[pos] = key_of(d_point_dist(xq, xf2 + 3 * (size_t)o), o);
            }
        }
        __syncwarp();
        const int seen = *cnt;
        if (seen > cap) {
            over = true;
            break;
        }
        if (seen >= K) {
            const unsigned long long kk = kth_key(keys, seen, K, lane);
            const float kd = __uint_as_float((unsigned)(kk >> 32));
            result = kk;  // best so far; the loop ends after the last ring anyway
            if (kd < __fsub_rn(__fmul_rn((float)r, pg.cell), pg.slack)) break;
        }
        __syncwarp();
    }
    __syncwarp();
    return !over;
}

// Pass 1: every kNN query with its keys in shared memory (kCap per warp); a
// query whose rings bring more points than that is appended to ovlist and
// redone by k_cand_kth_global.
__global__ void __launch_bounds__(kWarps * 32) k_cand_kth(DG pg, const float* __restrict__ xf1,
                                                         const float* __restrict__ xf2, int n1, int K_all, int self,
                                                         const int* __restrict__ qk,
                                                         unsigned long long* __restrict__ kth,
                                                         int* __restrict__ n_over, int* __restrict__ ovlist,
                                                         int qb0) {
    __shared__ unsigned long long keys[kWarps][kCap];
    __shared__ int cnt[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = gridDim.x * kWarps;
    for (int q = qb0 + blockIdx.x * kWarps + w; q < n1; q += nw) {
        const int K = qk ? qk[q] : K_all;
        if (K <= 0) continue;  // a within object of a mixed batch (warp-uniform)
        unsigned long long result;
        const bool ok = kth_search(pg, xf1 + 3 * (size_t)q, xf2, q, K, self, keys[w], kCap, &cnt[w], lane, result);
        if (lane == 0) {
            kth[q] = result;
            if (!ok) ovlist[atomicAdd(n_over, 1)] = q;
        }
        __syncwarp();
    }
}

// Pass 2, only when pass 1 overflowed: the queries of ovlist, one warp each,
// with a global-memory key buffer of cap (>= the points of tile 2) per warp.
__global__ void __launch_bounds__(kWarps * 32) k_cand_kth_global(DG pg, const float* __restrict__ xf1,
                                                                const float* __restrict__ xf2, int K_all, int self,
                                                                const int* __restrict__ qk,
                                                                unsigned long long* __restrict__ kth,
                                                                const int* __restrict__ n_over,
                                                                const int* __restrict__ ovlist,
                                                                unsigned long long* __restrict__ gkeys, int cap) {
    __shared__ int cnt[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarps + w, nw = gridDim.x * kWarps;
    unsigned long long* keys = gkeys + (size_t)gw * cap;
    for (int i = gw; i < *n_over; i += nw) {
        const int q = ovlist[i];
        const int K = qk ? qk[q] : K_all;
        unsigned long long result;
        kth_search(pg, xf1 + 3 * (size_t)q, xf2, q, K, self, keys, cap, &cnt[w], lane, result);
        if (lane == 0) kth[q] = result;
        __syncwarp();
    }
}

// first box-grid cell (the cell of its low corner) of every object of tile 2
__global__ void k_first_cells(DG bg, const float* __restrict__ box2, int n2, int4* __restrict__ fc) {
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n2; o += gridDim.x * blockDim.x) {
        const float* ob = box2 + 6 * (size_t)o;
        fc[o] = make_int4(dci(ob[0], bg.lo0, bg.cell, bg.n0), dci(ob[1], bg.lo1, bg.cell, bg.n1),
                          dci(ob[2], bg.lo2, bg.cell, bg.n2), 0);
    }
}

// The cells of the scan range are taken 32 at a time, one per lane; their
// item counts are prefix-summed across the warp and the lanes then stride
// over the items of all 32 cells together (each lane finds its item's cell by
// a binary search over the prefix), so a range of many sparse cells costs a
// few warp iterations instead of one per cell.
template <bool WRITE>
__global__ void __launch_bounds__(256) k_cand_pass(DG bg, const float* __restrict__ box1, const float* __restrict__ xf1,
                                                   const float* __restrict__ box2, const float* __restrict__ xf2,
                                                   const int4* __restrict__ fc, int n1, int self, int knn_all,
                                                   float tau_all, const int* __restrict__ qk,
                                                   const float* __restrict__ qtau, int isect,
                                                   const unsigned long long* __restrict__ kth,
                                                   int64_t* __restrict__ cnt, const int64_t* __restrict__ off,
                                                   unsigned long long* __restrict__ keys, int qb0, int qe0) {
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n1; q += nw) {
        if (q < qb0 || q >= qe0) {  // outside the joined query range: no candidates
            if (!WRITE && lane == 0) cnt[q] = 0;
            continue;
        }
        const float* qb = box1 + 6 * (size_t)q;
        const float* xq = xf1 + 3 * (size_t)q;
        const int knn = qk ? qk[q] > 0 : knn_all;
        const float tau = qk ? qtau[q] : tau_all;
        unsigned long long kk = 0;
        float T = tau;
        if (knn) {
            kk = kth[q];
            T = kk == ~0ull ? INFINITY : __uint_as_float((unsigned)(kk >> 32));
        }
        const float r = isinf(T) ? 3e38f : T;
        const int x0 = dci(__fsub_rn(qb[0], r), bg.lo0, bg.cell, bg.n0), x1 = dci(__fadd_rn(qb[3], r), bg.lo0, bg.cell, bg.n0);
        const int y0 = dci(__fsub_rn(qb[1], r), bg.lo1, bg.cell, bg.n1), y1 = dci(__fadd_rn(qb[4], r), bg.lo1, bg.cell, bg.n1);
        const int z0 = dci(__fsub_rn(qb[2], r), bg.lo2, bg.cell, bg.n2), z1 = dci(__fadd_rn(qb[5], r), bg.lo2, bg.cell, bg.n2);
        const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
        const int64_t ncell = (int64_t)(x1 - x0 + 1) * ny * nz;
        int64_t pos = WRITE ? off[q] : 0, count = 0;
        for (int64_t cb = 0; cb < ncell; cb += 32) {
            const int64_t L = cb + lane;
            int cx = 0, cy = 0, cz = 0;
            int64_t b = 0, n = 0;
            if (L < ncell) {
                cz = z0 + (int)(L % nz);
                const int64_t t = L / nz;
                cy = y0 + (int)(t % ny);
                cx = x0 + (int)(t / ny);
                const size_t c = ((size_t)cx * bg.n1 + cy) * bg.n2 + cz;
                b = bg.start[c];
                n = bg.start[c + 1] - b;
            }
            int64_t inc = n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t t = __shfl_up_sync(kFull, inc, o);
                if (lane >= o) inc += t;
            }
            const int64_t ex = inc - n;
            const int64_t tot = __shfl_sync(kFull, inc, 31);
            for (int64_t j0 = 0; j0 < tot; j0 += 32) {
                const int64_t j = j0 + lane;
                int k = 0;  // the last lane whose cell starts at or before item j
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (__shfl_sync(kFull, ex, k + step) <= j) k += step;
                const int64_t bk = __shfl_sync(kFull, b, k), ek = __shfl_sync(kFull, ex, k);
                const int xk = __shfl_sync(kFull, cx, k), yk = __shfl_sync(kFull, cy, k), zk = __shfl_sync(kFull, cz, k);
                bool keep = false;
                unsigned long long key = 0;
                if (j < tot) {
                    const int o = bg.items[bk + (j - ek)];
                    const float* ob = box2 + 6 * (size_t)o;
                    const int4 f = fc[o];
                    // count an object only in its first cell inside the scan range
                    if (max(f.x, x0) == xk && max(f.y, y0) == yk && max(f.z, z0) == zk && !(self && o == q)) {
                        const float gap = d_box_gap(ob, qb);
                        if (knn) {
                            const float md = d_point_dist(xq, xf2 + 3 * (size_t)o);
                            key = key_of(md, o);
                            keep = gap < T || key <= kk;
                        } else {
                            key = (unsigned)o;
                            keep = isect ? strict_overlap(ob, qb) : gap <= tau;
                        }
                    }
                }
                const unsigned m = __ballot_sync(kFull, keep);
                if (WRITE && keep) keys[pos + __popc(m & lt)] = key;
                pos += __popc(m);
                count += __popc(m);
            }
        }
        if (!WRITE && lane == 0) cnt[q] = count;
    }
}

__global__ void k_cand_finish(const int64_t* __restrict__ off, int n1, const unsigned long long* __restrict__ keys,
                              int* __restrict__ pq, int* __restrict__ pt) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n1; q += gridDim.x * blockDim.x)
        for (int64_t k = off[q]; k < off[q + 1]; ++k) {
            pq[k] = q;
            pt[k] = (int)(keys[k] & 0xffffffffull);
        }
}

int upload_grid(tdp_ctx* ctx, DevGrid& g, const CellGrid& h) {
    for (int k = 0; k < 3; ++k) {
        g.lo[k] = h.lo[k];
        g.n[k] = h.n[k];
    }
    g.cell = h.cell;
    g.slack = h.slack;
    // from the block cache (at least a cached block's size): a tile attached
    // and freed every request then neither allocates nor frees device memory
    if (block_alloc(ctx, (void**)&g.start, std::max<size_t>(h.start.size() * 8, kCachedBlockMin)) != cudaSuccess ||
        block_alloc(ctx, (void**)&g.items, std::max<size_t>(h.items.size() * 4, kCachedBlockMin)) != cudaSuccess)
        return fail(ctx, TDP_ERR_NOMEM, "cannot allocate the candidate grid");
    cudaMemcpyAsync(g.start, h.start.data(), h.start.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (!h.items.empty())
        cudaMemcpyAsync(g.items, h.items.data(), h.items.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
    g.ready = true;
    return TDP_OK;
}

// Device copies of the host boxes and transforms of a tile (cached in the grid record).
struct TileBoxes {
    float* box = nullptr;
    float* xf = nullptr;
};

}  // namespace

int device_candidates(tdp_ctx* ctx, const tdp_tile* t1, const tdp_tile* t2, bool self, bool knn, int K, float tau,
                      Buf& pq_buf, Buf& pt_buf, Buf& qoff_buf, long& P, long& n_redone, const int* qk,
                      const float* qtau, bool isect, long q_begin, long q_end) {
    cudaStream_t s = ctx->stream;
    const long n1 = t1->n_obj, n2 = t2->n_obj;
    const long qb0 = std::max(0L, q_begin), qe0 = q_end < 0 ? n1 : std::min(n1, q_end);
    n_redone = 0;
    P = 0;
    int rc;
    // grids over tile 2, built once per tile
    if (!t2->box_grid.ready) {
        const float cell = pick_cell(t2->host.obj_box.data(), n2);
        CellGrid hb;
        hb.build(t2->host.obj_box.data(), n2, 6, 3, cell);
        if ((rc = upload_grid(ctx, t2->box_grid, hb))) return rc;
        CellGrid hp;
        hp.build(t2->host.obj_xf.data(), n2, 3, 0, cell);
        if ((rc = upload_grid(ctx, t2->point_grid, hp))) return rc;
    }
    // device copies of both tiles' boxes and transforms
    Buf& kthb = ctx->scratch[52];
    Buf& cntb = ctx->scratch[53];
    Buf& keys = ctx->scratch[54];
    Buf& keys2 = ctx->scratch[55];
    Buf& tmp = ctx->scratch[56];
    if ((rc = ensure(ctx, kthb, (size_t)(n1 + 1) * 8))) return rc;
    if ((rc = ensure(ctx, cntb, (size_t)(n1 + 1) * 8))) return rc;
    if ((rc = ensure(ctx, qoff_buf, (size_t)(n1 + 1) * 8))) return rc;
#define CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)
    // the tiles' boxes and transforms stay on the device between joins
    for (const tdp_tile* t : {t1, t2}) {
        if (t->d_boxes && t->boxes_n == t->n_obj) continue;
        dfree(ctx, t->d_boxes);
        t->d_boxes = nullptr;
        if (block_alloc(ctx, (void**)&t->d_boxes, (size_t)std::max<long>(t->n_obj, 1) * 9 * 4) != cudaSuccess)
            return fail(ctx, TDP_ERR_NOMEM, "cannot allocate the candidate boxes");
        CU(cudaMemcpyAsync(t->d_boxes, t->host.obj_box.data(), t->n_obj * 24, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(t->d_boxes + 6 * t->n_obj, t->host.obj_xf.data(), t->n_obj * 12, cudaMemcpyHostToDevice,
                           s));
        t->boxes_n = t->n_obj;
    }
    const float* box1 = t1->d_boxes;
    const float* xf1 = box1 + 6 * n1;
    const float* box2 = t2->d_boxes;
    const float* xf2 = box2 + 6 * n2;
    int* d_over = (int*)(ctx->d_counter + 40);
    Buf& ovb = ctx->scratch[89];
    if ((rc = ensure(ctx, ovb, (size_t)(n1 + 1) * 4))) return rc;
    CU(cudaMemsetAsync(d_over, 0, 4, s));
    const DG bg = dg(t2->box_grid), pg = dg(t2->point_grid);
    unsigned long long* kth = (unsigned long long*)kthb.p;
    const bool any_knn = knn || qk;
    if (any_knn) {
        const long nq = std::max(0L, qe0 - qb0);
        const int blocks = (int)std::min<long>((nq + kWarps - 1) / kWarps, (long)ctx->num_sms * 16);
        k_cand_kth<<<std::max(blocks, 1), kWarps * 32, 0, s>>>(pg, xf1, xf2, (int)qe0, K, self, qk, kth, d_over,
                                                              (int*)ovb.p, (int)qb0);
        CU(cudaGetLastError());
    }
    // first cell of every tile-2 object (the dedupe test of the scan)
    Buf& fcb = ctx->scratch[88];
    if ((rc = ensure(ctx, fcb, (size_t)std::max<long>(n2, 1) * sizeof(int4)))) return rc;
    const int4* fc = (const int4*)fcb.p;
    k_first_cells<<<(int)std::max<long>(1, std::min<long>((n2 + 255) / 256, (long)ctx->num_sms * 8)), 256, 0, s>>>(
        bg, box2, (int)n2, (int4*)fcb.p);
    CU(cudaGetLastError());
    int64_t* cnt = (int64_t*)cntb.p;
    int64_t* qoff = (int64_t*)qoff_buf.p;
    const int pblocks = (int)std::min<long>((n1 + 7) / 8, (long)ctx->num_sms * 32);
    int64_t total = 0;
    int over = 0;
    for (int pass = 0;; ++pass) {
        CU(cudaMemsetAsync(cnt + n1, 0, 8, s));
        k_cand_pass<false><<<std::max(pblocks, 1), 256, 0, s>>>(bg, box1, xf1, box2, xf2, fc, (int)n1, self, knn, tau,
                                                               qk, qtau, isect ? 1 : 0, kth, cnt, nullptr, nullptr,
                                                               (int)qb0, (int)qe0);
        CU(cudaGetLastError());
        size_t tb = 0;
        CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, qoff, (int)n1 + 1, s));
        if ((rc = ensure(ctx, tmp, tb + 16))) return rc;
        CU(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt, qoff, (int)n1 + 1, s));
        CU(cudaMemcpyAsync(&total, qoff + n1, 8, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(&over, d_over, 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (!over || pass > 0) break;
        // Some kNN ring searches saw more points than a warp's shared-memory
        // buffer holds: redo just those on the device with a global buffer of
        // n2 + 1 keys per warp (which no ring search can overflow), then count
        // again.  At most 256 MiB of keys, at least one warp.
        const long cap = n2 + 1;
        const long warps = std::max<long>(1, std::min<long>({(long)over, (long)ctx->num_sms * kWarps,
                                                             (256L << 20) / (cap * 8)}));
        Buf& gk = ctx->scratch[90];
        if ((rc = ensure(ctx, gk, (size_t)warps * cap * 8))) return rc;
        k_cand_kth_global<<<(int)((warps + kWarps - 1) / kWarps), kWarps * 32, 0, s>>>(
            pg, xf1, xf2, K, self, qk, kth, d_over, (const int*)ovb.p, (unsigned long long*)gk.p, (int)cap);
        CU(cudaGetLastError());
        n_redone = over;
    }
    if (total >= (1LL << 31) - 1) return fail(ctx, TDP_ERR_ARG, "too many candidate pairs");
    P = (long)total;
    const size_t Pz = (size_t)std::max<long>(P, 1);
    if ((rc = ensure(ctx, keys, Pz * 8))) return rc;
    if ((rc = ensure(ctx, keys2, Pz * 8))) return rc;
    if ((rc = ensure(ctx, pq_buf, Pz * 4))) return rc;
    if ((rc = ensure(ctx, pt_buf, Pz * 4))) return rc;
    if (P > 0) {
        k_cand_pass<true><<<std::max(pblocks, 1), 256, 0, s>>>(bg, box1, xf1, box2, xf2, fc, (int)n1, self, knn, tau, qk, qtau, isect ? 1 : 0, kth,
                                                              nullptr, qoff, (unsigned long long*)keys.p, (int)qb0,
                                                              (int)qe0);
        CU(cudaGetLastError());
        size_t sb = 0;
        CU(cub::DeviceSegmentedSort::SortKeys(nullptr, sb, (const unsigned long long*)keys.p,
                                              (unsigned long long*)keys2.p, (int)P, (int)n1, qoff, qoff + 1, s));
        if ((rc = ensure(ctx, tmp, sb + 16))) return rc;
        CU(cub::DeviceSegmentedSort::SortKeys(tmp.p, sb, (const unsigned long long*)keys.p,
                                              (unsigned long long*)keys2.p, (int)P, (int)n1, qoff, qoff + 1, s));
        const int fblocks = (int)std::min<long>((n1 + 255) / 256, (long)ctx->num_sms * 8);
        k_cand_finish<<<std::max(fblocks, 1), 256, 0, s>>>(qoff, (int)n1, (const unsigned long long*)keys2.p,
                                                          (int*)pq_buf.p, (int*)pt_buf.p);
        CU(cudaGetLastError());
    }
#undef CU
    return TDP_OK;
}

}  // namespace tdp

extern "C" long tdp_tile_candidates(tdp_ctx* ctx, const tdp_tile* t1, const tdp_tile* t2, int is_knn, int knn,
                                    float within, int64_t* off, int32_t* ids, long cap) {
    using namespace tdp;
    if (!ctx || !t1 || !off || (is_knn && knn < 1)) return LONG_MIN;
    const bool self = (t2 == nullptr || t2 == t1);
    if (!t2) t2 = t1;
    cudaSetDevice(ctx->device);
    long P = 0, redone = 0;
    Buf& pq = ctx->scratch[57];
    Buf& pt = ctx->scratch[58];
    Buf& qo = ctx->scratch[59];
    if (device_candidates(ctx, t1, t2, self, is_knn != 0, is_knn ? knn : 0, within, pq, pt, qo, P, redone))
        return LONG_MIN;
    ctx->stats.candidate_redone = redone;
    cudaMemcpyAsync(off, qo.p, (t1->n_obj + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (ids && P <= cap && P > 0) cudaMemcpyAsync(ids, pt.p, P * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return LONG_MIN;
    return (P > cap || !ids) ? -P : P;
}
