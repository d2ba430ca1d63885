// bounds_kernels.cu -- GPU preparation of the per-triangle Hausdorff bounds of a
// resident tile (tdp_tile_compute_bounds).
//
// Replaces the reference's CGAL preparation of the bounds that the join reads
// (sampling in src/spatial/himesh_hausdorff.cpp:197-270; stored per triangle as
// (proxy, hausdorff) at src/spatial/himesh_retrieve.cpp:131-151 and consumed by
// the refine at src/geometry/computing_gpu.cu:1115-1117) with a conservative
// rule evaluated in FP64 from each object's own LOD-100 surface S:
//   ph(t): each LOD-100 facet s is assigned to the LOD-l triangle t nearest its
//          barycentre (ties to the lower index); ph(t) = max over assigned s
//          and the vertices q of s of dist(q, t).  dist(., t) is convex, so
//          every point of s lies within ph(t) of t: d(t1, t2) - ph1 - ph2 is a
//          lower bound of the LOD-100 distance.
//   h(t):  t is cut by d midpoint subdivisions (d = least of 0..3 with
//          longest edge / 2^d <= 1.5 x the mean LOD-100 edge of the object) and
//          h(t) = max over pieces of min over s of max over the piece's corners
//          of dist(corner, s).  By convexity of dist(., s) every point of t lies
//          within h(t) of S: d(t1, t2) + h1 + h2 is an upper bound.
// Both round up to float; the object-level values are the per-LOD maxima.
//
// Layout of the work: one warp per (LOD, voxel) item.  A facet's nearest
// triangle is searched in its own voxel first, then in every other voxel of the
// object whose box (of that LOD's triangles) is within the best distance so far
// plus a margin far above FP64 rounding, lanes striding over the voxel's
// triangles, a lexicographic (distance, index) warp minimum after each voxel.
// The pieces' nearest facets are searched the same way with each lane cutting a
// facet short once its running maximum reaches the best value.  Distances are
// compared squared and rooted once per result (sqrt is monotone and correctly
// rounded, so this changes no bound); the nearest-triangle assignment breaks
// ties on the squared distance.  Both searches
// return exactly what a scan of every triangle returns.  This file is built
// with -fmad=false: each product and sum is rounded on its own, so the FP64
// values equal a host evaluation of the same expressions.
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstring>
#include <string>

#include "ctx.cuh"
#include "bounds_kernels.cuh"
#include "fetch_kernels.cuh"
#include "ptdist.cuh"
#include "storage/dev_tile.h"

namespace tdp {
namespace {

using pd::D3;

constexpr int kBoundsThreads = 256;
constexpr int kBoundsBlocksPerSm = 2;
enum BoundSlot { kBoxes = 84, kVobj, kMeanEdge, kBoundCounters };

struct BoundsDev {
    const float4* tri[kNumLods];
    const uint32_t* vtri[kNumLods];
    const float4* box[kNumLods];  // per voxel: (lo, 0), (hi, 0) of its triangles at that LOD
    const uint32_t* obj_vox;
    const int* vobj;
    const double* e0;
    long n_vox, n_obj;
    unsigned long long* counters;  // [0] distance evaluations, [1] facet queries, [2] pieces
};

__device__ inline D3 vert(const float4* tri, size_t t, int k) {
    const float4 v = tri[3 * t + k];
    return D3{(double)v.x, (double)v.y, (double)v.z};
}

__device__ inline void warp_min_idx(double& d, unsigned& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, d, o);
        const unsigned oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (od < d || (od == d && oi < i)) { d = od; i = oi; }
    }
}

__device__ inline double warp_min(double d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = pd::dmin(d, __shfl_xor_sync(0xffffffffu, d, o));
    return d;
}

__device__ inline unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// zero the (proxy, hausdorff) fields of every triangle record of one LOD
__global__ void k_zero_bounds(float4* tri, size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        tri[3 * t].w = 0.f;
        tri[3 * t + 1].w = 0.f;
    }
}

// box of every voxel's triangles at one LOD (+inf/-inf for an empty voxel)
__global__ void k_voxel_boxes(const float4* __restrict__ tri, const uint32_t* __restrict__ vtri, long n_vox,
                              float4* __restrict__ box) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < n_vox; v += (long)gridDim.x * blockDim.x) {
        float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        for (uint32_t t = vtri[v]; t < vtri[v + 1]; ++t)
            for (int k = 0; k < 3; ++k) {
                const float4 p = tri[3 * (size_t)t + k];
                lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
                hi.x = fmaxf(hi.x, p.x); hi.y = fmaxf(hi.y, p.y); hi.z = fmaxf(hi.z, p.z);
            }
        box[2 * v] = lo;
        box[2 * v + 1] = hi;
    }
}

// object of every voxel; mean LOD-100 edge length of every object (its facets
// and their edges (0,1), (1,2), (2,0) summed in stored order)
__global__ void k_objects(BoundsDev b, int* vobj, double* e0) {
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < b.n_obj; o += (long)gridDim.x * blockDim.x) {
        const uint32_t vb = b.obj_vox[o], ve = b.obj_vox[o + 1];
        for (uint32_t v = vb; v < ve; ++v) vobj[v] = (int)o;
        const uint32_t s0 = b.vtri[4][vb], s1 = b.vtri[4][ve];
        double sum = 0;
        for (uint32_t s = s0; s < s1; ++s) {
            const D3 p = vert(b.tri[4], s, 0), q = vert(b.tri[4], s, 1), r = vert(b.tri[4], s, 2);
            sum = sum + pd::dist(p, q);
            sum = sum + pd::dist(q, r);
            sum = sum + pd::dist(r, p);
        }
        e0[o] = s1 > s0 ? sum / (3.0 * (double)(s1 - s0)) : 0.0;
    }
}

// ph: every LOD-100 facet of voxel v -> nearest LOD-l triangle; raise that
// triangle's proxy bound to the facet's farthest vertex distance
__global__ void __launch_bounds__(kBoundsThreads, kBoundsBlocksPerSm) k_proxy(BoundsDev b) {
    const int lane = threadIdx.x & 31;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long evals = 0, queries = 0;
    for (long it = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < 4 * b.n_vox; it += warps) {
        const int l = (int)(it / b.n_vox);
        const long v = it - (long)l * b.n_vox;
        const int o = b.vobj[v];
        const uint32_t vb = b.obj_vox[o], ve = b.obj_vox[o + 1];
        const float4* T = b.tri[l];
        const uint32_t* VT = b.vtri[l];
        if (VT[vb] == VT[ve]) continue;  // the object has no triangle at this LOD
        const float4* box = b.box[l];
        const float4* S = b.tri[4];
        for (uint32_t s = b.vtri[4][v]; s < b.vtri[4][v + 1]; ++s) {
            const D3 a = vert(S, s, 0), c1 = vert(S, s, 1), c2 = vert(S, s, 2);
            const D3 q{(a.x + c1.x + c2.x) * (1.0 / 3.0), (a.y + c1.y + c2.y) * (1.0 / 3.0),
                       (a.z + c1.z + c2.z) * (1.0 / 3.0)};
            const double eps = pd::margin(q);
            double bd = INFINITY;  // squared distance of the nearest triangle so far
            unsigned bi = UINT_MAX;
            auto visit = [&](uint32_t u) {
                for (uint32_t t = VT[u] + lane; t < VT[u + 1]; t += 32) {
                    const double d = pd::tri2(q, vert(T, t, 0), vert(T, t, 1), vert(T, t, 2));
                    ++evals;
                    if (d < bd || (d == bd && t < bi)) { bd = d; bi = t; }
                }
                warp_min_idx(bd, bi);
            };
            visit((uint32_t)v);
            for (uint32_t base = vb; base < ve; base += 32) {
                const uint32_t u = base + lane;
                const bool cand = u < ve && u != (uint32_t)v;
                const double lb = cand ? pd::box_gap(q, box[2 * (size_t)u], box[2 * (size_t)u + 1]) : INFINITY;
                unsigned mask = __ballot_sync(0xffffffffu, cand && lb <= sqrt(bd) + eps);
                while (mask) {
                    const int k = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const double lbk = __shfl_sync(0xffffffffu, lb, k);
                    if (lbk <= sqrt(bd) + eps) visit(base + k);
                }
            }
            if (lane == 0) ++queries;
            if (bi == UINT_MAX) continue;
            double m = 0;
            if (lane < 3) {
                m = pd::tri2(vert(S, s, lane), vert(T, bi, 0), vert(T, bi, 1), vert(T, bi, 2));
                ++evals;
            }
            m = pd::dmax(m, __shfl_down_sync(0xffffffffu, m, 1));
            m = pd::dmax(m, __shfl_down_sync(0xffffffffu, m, 2));
            if (lane == 0)
                atomicMax(reinterpret_cast<unsigned*>(const_cast<float*>(&T[3 * (size_t)bi].w)),
                          __float_as_uint(__double2float_ru(sqrt(m))));
        }
    }
    evals = warp_sum(evals);
    if (lane == 0) {
        atomicAdd(&b.counters[0], evals);
        atomicAdd(&b.counters[1], queries);
    }
}

// h: every LOD-l triangle of voxel v, cut into pieces, each piece's nearest
// LOD-100 facet by the largest corner distance
__global__ void __launch_bounds__(kBoundsThreads, kBoundsBlocksPerSm) k_hausdorff(BoundsDev b) {
    const int lane = threadIdx.x & 31;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long evals = 0, npieces = 0;
    for (long it = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < 4 * b.n_vox; it += warps) {
        const int l = (int)(it / b.n_vox);
        const long v = it - (long)l * b.n_vox;
        const int o = b.vobj[v];
        const uint32_t vb = b.obj_vox[o], ve = b.obj_vox[o + 1];
        const float4* T = b.tri[l];
        const float4* S = b.tri[4];
        const uint32_t* VS = b.vtri[4];
        const float4* box = b.box[4];
        const bool has_s = VS[vb] != VS[ve];
        const double e0 = b.e0[o];
        unsigned seed = UINT_MAX;
        for (uint32_t t = b.vtri[l][v]; t < b.vtri[l][v + 1]; ++t) {
            const D3 a = vert(T, t, 0), c1 = vert(T, t, 1), c2 = vert(T, t, 2);
            const double L = pd::dmax(pd::dist(a, c1), pd::dmax(pd::dist(c1, c2), pd::dist(c2, a)));
            int dep = 0;
            while (dep < 3 && L / (double)(1 << dep) > 1.5 * e0) ++dep;
            double h = 0;
            const int np = has_s ? 1 << (2 * dep) : 0;
            for (int p = 0; p < np; ++p) {
                D3 w0{1, 0, 0}, w1{0, 1, 0}, w2{0, 0, 1};
                for (int lvl = 0; lvl < dep; ++lvl) {
                    const int ch = (p >> (2 * (dep - 1 - lvl))) & 3;
                    const D3 m01{(w0.x + w1.x) * 0.5, (w0.y + w1.y) * 0.5, (w0.z + w1.z) * 0.5};
                    const D3 m12{(w1.x + w2.x) * 0.5, (w1.y + w2.y) * 0.5, (w1.z + w2.z) * 0.5};
                    const D3 m20{(w2.x + w0.x) * 0.5, (w2.y + w0.y) * 0.5, (w2.z + w0.z) * 0.5};
                    if (ch == 0) { w1 = m01; w2 = m20; }
                    else if (ch == 1) { w0 = w1; w1 = m12; w2 = m01; }
                    else if (ch == 2) { w0 = w2; w1 = m20; w2 = m12; }
                    else { w0 = m01; w1 = m12; w2 = m20; }
                }
                const D3 W[3] = {w0, w1, w2};
                D3 q[3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    q[k] = D3{a.x * W[k].x + c1.x * W[k].y + c2.x * W[k].z, a.y * W[k].x + c1.y * W[k].y + c2.y * W[k].z,
                              a.z * W[k].x + c1.z * W[k].y + c2.z * W[k].z};
                const double eps = pd::dmax(pd::margin(q[0]), pd::dmax(pd::margin(q[1]), pd::margin(q[2])));
                // seed: the previous piece's nearest facet (a neighbour of this
                // piece) bounds the minimum before the scan, so most facets of
                // the scan stop after their first corner
                double best = INFINITY;
                unsigned best_i = UINT_MAX;
                if (seed != UINT_MAX) {
                    double dk = 0;
                    if (lane < 3) {
                        const D3 qk = lane == 0 ? q[0] : (lane == 1 ? q[1] : q[2]);
                        dk = pd::tri2(qk, vert(S, seed, 0), vert(S, seed, 1), vert(S, seed, 2));
                        ++evals;
                    }
                    dk = pd::dmax(dk, __shfl_down_sync(0xffffffffu, dk, 1));
                    dk = pd::dmax(dk, __shfl_down_sync(0xffffffffu, dk, 2));
                    best = __shfl_sync(0xffffffffu, dk, 0);
                    best_i = seed;
                }
                auto visit = [&](uint32_t u) {
                    double mine = best;
                    unsigned mi = best_i;
                    for (uint32_t s = VS[u] + lane; s < VS[u + 1]; s += 32) {
                        const D3 sa = vert(S, s, 0), sb = vert(S, s, 1), sc = vert(S, s, 2);
                        double acc = 0;
                        bool whole = true;
#pragma unroll 1
                        for (int k = 0; k < 3; ++k) {
                            acc = pd::dmax(acc, pd::tri2(q[k], sa, sb, sc));
                            ++evals;
                            if (acc >= mine) { whole = k == 2; break; }
                        }
                        if (whole && acc < mine) { mine = acc; mi = s; }
                    }
                    warp_min_idx(mine, mi);
                    best = mine;
                    best_i = mi;
                };
                visit((uint32_t)v);
                for (uint32_t base = vb; base < ve; base += 32) {
                    const uint32_t u = base + lane;
                    const bool cand = u < ve && u != (uint32_t)v;
                    double lb = INFINITY;
                    if (cand) {
                        const float4 lo = box[2 * (size_t)u], hi = box[2 * (size_t)u + 1];
                        lb = pd::dmax(pd::box_gap(q[0], lo, hi), pd::dmax(pd::box_gap(q[1], lo, hi), pd::box_gap(q[2], lo, hi)));
                    }
                    unsigned mask = __ballot_sync(0xffffffffu, cand && lb <= sqrt(best) + eps);
                    while (mask) {
                        const int k = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const double lbk = __shfl_sync(0xffffffffu, lb, k);
                        if (lbk <= sqrt(best) + eps) visit(base + k);
                    }
                }
                h = pd::dmax(h, best);
                seed = best_i;
            }
            if (lane == 0) {
                const_cast<float4*>(T)[3 * (size_t)t + 1].w = __double2float_ru(sqrt(h));
                npieces += np;
            }
        }
    }
    evals = warp_sum(evals);
    if (lane == 0) {
        atomicAdd(&b.counters[0], evals);
        atomicAdd(&b.counters[2], npieces);
    }
}

// object-level values: per LOD the largest hausdorff and proxy bound (0 at LOD 100)
__global__ void k_object_bounds(BoundsDev b, float* obj_hd, float* obj_phd) {
    const int lane = threadIdx.x & 31;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long it = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < kNumLods * b.n_obj; it += warps) {
        const long o = it / kNumLods;
        const int l = (int)(it - o * kNumLods);
        float mh = 0.f, mp = 0.f;
        if (l < kNumLods - 1) {
            const uint32_t t0 = b.vtri[l][b.obj_vox[o]], t1 = b.vtri[l][b.obj_vox[o + 1]];
            for (uint32_t t = t0 + lane; t < t1; t += 32) {
                mp = fmaxf(mp, b.tri[l][3 * (size_t)t].w);
                mh = fmaxf(mh, b.tri[l][3 * (size_t)t + 1].w);
            }
#pragma unroll
            for (int k = 16; k > 0; k >>= 1) {
                mp = fmaxf(mp, __shfl_xor_sync(0xffffffffu, mp, k));
                mh = fmaxf(mh, __shfl_xor_sync(0xffffffffu, mh, k));
            }
        }
        if (lane == 0) {
            obj_hd[o * kNumLods + l] = mh;
            obj_phd[o * kNumLods + l] = mp;
        }
    }
}

__global__ void k_gather_bounds(const float4* __restrict__ tri, size_t n, float2* __restrict__ out) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        out[t] = make_float2(tri[3 * t].w, tri[3 * t + 1].w);
}

}  // namespace

cudaError_t launch_gather_bounds(const float4* tri, size_t n, float* out, cudaStream_t s) {
    if (!n) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_gather_bounds<<<sms * 8, 256, 0, s>>>(tri, n, reinterpret_cast<float2*>(out));
    return cudaGetLastError();
}

}  // namespace tdp

using namespace tdp;

extern "C" int tdp_tile_compute_bounds(tdp_ctx* ctx, tdp_tile* tile, tdp_bounds_info* info) {
    if (!ctx || !tile) return TDP_ERR_ARG;
    if (tile->device != ctx->device) return fail(ctx, TDP_ERR_ARG, "tile lives on another device");
    if (info) std::memset(info, 0, sizeof(*info));
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const long nv = tile->n_vox, no = tile->n_obj;
    if (no == 0 || nv == 0) return TDP_OK;
    int rc;
    if ((rc = ensure(ctx, ctx->scratch[kBoxes], (size_t)kNumLods * nv * 2 * sizeof(float4)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kVobj], (size_t)nv * sizeof(int)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kMeanEdge], (size_t)no * sizeof(double)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kBoundCounters], 4 * sizeof(unsigned long long)))) return rc;
    BoundsDev b{};
    float4* boxes = (float4*)ctx->scratch[kBoxes].p;
    for (int l = 0; l < kNumLods; ++l) {
        b.tri[l] = tile->tri[l];
        b.vtri[l] = tile->vtri[l];
        b.box[l] = boxes + (size_t)l * nv * 2;
    }
    b.obj_vox = tile->obj_vox;
    b.vobj = (const int*)ctx->scratch[kVobj].p;
    b.e0 = (const double*)ctx->scratch[kMeanEdge].p;
    b.n_vox = nv;
    b.n_obj = no;
    b.counters = (unsigned long long*)ctx->scratch[kBoundCounters].p;
#define CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)
    // an attached tile first fetches every voxel: the bounds are written into
    // the device records, which later fetches must not overwrite
    CU(launch_fetch_all(lazy_view(tile), ctx->num_sms, s));
    CU(cudaEventRecord(ctx->ev[0], s));
    CU(cudaMemsetAsync(b.counters, 0, 4 * sizeof(unsigned long long), s));
    const int small_grid = ctx->num_sms * 8;
    for (int l = 0; l < kNumLods; ++l) {
        const size_t n = tile->host.n_tris[l];
        if (n) k_zero_bounds<<<small_grid, 256, 0, s>>>(tile->tri[l], n);
        k_voxel_boxes<<<small_grid, 128, 0, s>>>(tile->tri[l], tile->vtri[l], nv, boxes + (size_t)l * nv * 2);
    }
    k_objects<<<(int)((no + 127) / 128), 128, 0, s>>>(b, (int*)ctx->scratch[kVobj].p, (double*)ctx->scratch[kMeanEdge].p);
    const int grid = ctx->num_sms * kBoundsBlocksPerSm;
    k_proxy<<<grid, kBoundsThreads, 0, s>>>(b);
    k_hausdorff<<<grid, kBoundsThreads, 0, s>>>(b);
    k_object_bounds<<<small_grid, 256, 0, s>>>(b, tile->obj_hd, tile->obj_phd);
    CU(cudaGetLastError());
    CU(cudaEventRecord(ctx->ev[1], s));
    unsigned long long cnt[4] = {0, 0, 0, 0};
    CU(cudaMemcpyAsync(cnt, b.counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    tile->host.obj_hd.resize((size_t)no * kNumLods);
    tile->host.obj_phd.resize((size_t)no * kNumLods);
    CU(cudaMemcpyAsync(tile->host.obj_hd.data(), tile->obj_hd, (size_t)no * kNumLods * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(tile->host.obj_phd.data(), tile->obj_phd, (size_t)no * kNumLods * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
#undef CU
    if (info) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        info->ms = ms;
        info->objects = no;
        long tris = 0;
        for (int l = 0; l < kNumLods - 1; ++l) tris += (long)tile->host.n_tris[l];
        info->triangles = tris;
        info->dist_evals = (double)cnt[0];
        info->facet_queries = (long)cnt[1];
        info->pieces = (long)cnt[2];
    }
    return TDP_OK;
}
