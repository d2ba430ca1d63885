// exact_kernels.cu -- exact (FP64) distances of the join's reported pairs.
//
// The reference reports result ids only (HiMesh_Wrapper::report_result,
// src/spatial/himesh_wrapper.cpp:195-202); a pair decided before LOD 100 has
// only a Hausdorff-widened range.  When tdp_join_params.exact_distances is set,
// this stage gives every reported pair its LOD-100 distance in FP64:
//   1. U, an upper bound of the pair's LOD-100 distance D: the smallest
//      core-to-core distance over its voxel pairs (a core is a vertex of the
//      LOD-100 surface), and, at Hausdorff level 2, also the pair's upper
//      bound pmx when it was decided (d + h1 + h2 at a lower LOD bounds D);
//      each widened by its FP32 error, max(perr, 1e-4 (value + 1));
//      U is then tightened by refining, in FP32, the voxel pair with the
//      closest cores (kExK per object pair): its minimum d32 + err_bound(R)
//      is a distance between two surface points, hence also >= D;
//   2. every LOD-100 voxel pair whose box gap is <= U is a candidate (the
//      voxel pair holding the closest points has gap <= D <= U);
//   3. the tuned FP32 refine, its minimum preset to U plus the candidate's
//      largest possible FP32 error, gives each candidate that has a triangle
//      pair below that preset its minimum d32 (error e = err_bound(R)) and
//      skips the rest after a few cluster tests (sphere and cylinder bounds);
//      per object pair best32 =
//      min d32 and E = max e;
//   4. a candidate can hold the minimum only if d32 - E <= best32 + E (its
//      true minimum is >= d32 - e, and D <= best32 + E): those are evaluated
//      again triangle pair by triangle pair, skipping pairs whose (inflated)
//      bounding-sphere gap or cylinder bound exceeds best32 + 2E; a pair's
//      FP32 distance d32'
//      with its error e' comes first, and only a pair with d32' - e' <=
//      best32 + E (one that can be the minimum) is evaluated in FP64;
//   5. D = the smallest FP64 distance over the evaluated candidates.
// Every filter is conservative, so D is the exact minimum over the stored
// float coordinates up to the FP64 rounding of one triangle distance.
#include <cub/device/device_scan.cuh>
#include <float.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "exact_kernels.cuh"
#include "cull.cuh"
#include "refine.cuh"
#include "tridist.cuh"

namespace tdp {
namespace {

constexpr int kBlk = 256;

// Voxel pairs per object pair refined in FP32 to tighten U (the ones with
// the closest cores).  On the within-400 join eight cost 8x the FP32 work of
// one and left the candidate set 1.4 % smaller (28.0 M voxel pairs against
// 28.4 M); the two with the smallest box gaps instead gave a looser U (29.6 M
// candidates, 15 % more FP32 work); so one is refined.
constexpr int kExK = 1;

// The FP32 passes run the lazy refine with the cylinder bound in its culls
// (configuration 16): a reported pair's closest points face each other across
// a gap of up to tau, where the sphere gap keeps every triangle pair whose
// centres are offset sideways by less than about sqrt(2 gap (r1 + r2)).
constexpr int kExactRefineCfg = 16;

// U of every reported pair: min core-to-core distance over its voxel pairs,
// and pmx when it is a proven bound (pmx_valid); item1[kExK p + k] = the voxel
// pairs with the kExK closest cores (empty items for the rest and for pairs
// that are not reported).  Each lane keeps a sorted top kExK of its own
// (strided) voxel pairs; the warp then takes the kExK smallest heads.
__global__ void __launch_bounds__(kBlk) k_exact_upper(JoinDev d, int pmx_valid, const uint32_t* __restrict__ vt1,
                                                      const uint32_t* __restrict__ vt2, float* __restrict__ U,
                                                      RefineItem* __restrict__ item1) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        RefineItem* it1 = item1 + (size_t)kExK * p;
        if (d.pstat[p] != kReported) {
            if (lane == 0) U[p] = FLT_MAX;
            if (lane < kExK) it1[lane] = RefineItem{0, 0, 0, 0};
            continue;
        }
        const int q = d.pq[p], t = d.pt[p];
        const uint32_t a0 = d.ovox1[q], a1 = d.ovox1[q + 1], b0 = d.ovox2[t], b1 = d.ovox2[t + 1];
        float kv[kExK];
        uint32_t ka[kExK], kb[kExK];
#pragma unroll
        for (int k = 0; k < kExK; ++k) { kv[k] = FLT_MAX; ka[k] = a0; kb[k] = b0; }
        for (uint32_t b = b0 + lane; b < b1; b += 32) {
            if (vt2[b + 1] == vt2[b]) continue;
            const float4 cb = d.vox2[3 * (size_t)b + 2];
            for (uint32_t a = a0; a < a1; ++a) {
                if (vt1[a + 1] == vt1[a]) continue;
                const float4 ca = d.vox1[3 * (size_t)a + 2];
                const float dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
                float v = dx * dx + dy * dy + dz * dz;
                if (!(v < kv[kExK - 1])) continue;
                // insert into the lane's sorted list (unrolled, registers only)
                uint32_t ia = a, ib = b;
#pragma unroll
                for (int k = 0; k < kExK; ++k) {
                    if (v < kv[k]) {
                        const float tv = kv[k];
                        const uint32_t ta = ka[k], tb = kb[k];
                        kv[k] = v; ka[k] = ia; kb[k] = ib;
                        v = tv; ia = ta; ib = tb;
                    }
                }
            }
        }
        // the warp's kExK smallest: each round takes the smallest lane head
        float best = FLT_MAX;
        for (int k = 0; k < kExK; ++k) {
            float h = kv[0];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) h = fminf(h, __shfl_xor_sync(0xffffffffu, h, o));
            const unsigned who = __ballot_sync(0xffffffffu, kv[0] == h);
            const int src = __ffs(who) - 1;
            const uint32_t wa = __shfl_sync(0xffffffffu, ka[0], src), wb = __shfl_sync(0xffffffffu, kb[0], src);
            if (k == 0) best = h;
            if (lane == 0)
                it1[k] = h < FLT_MAX ? RefineItem{vt1[wa], vt1[wa + 1] - vt1[wa], vt2[wb], vt2[wb + 1] - vt2[wb]}
                                     : RefineItem{0, 0, 0, 0};
            if (lane == src) {  // pop the head
#pragma unroll
                for (int j = 0; j + 1 < kExK; ++j) { kv[j] = kv[j + 1]; ka[j] = ka[j + 1]; kb[j] = kb[j + 1]; }
                kv[kExK - 1] = FLT_MAX;
            }
        }
        if (lane == 0) {
            float u = FLT_MAX;
            if (best < FLT_MAX) {
                const float core = sqrtf(best);
                u = core + fmaxf(1e-4f * (core + 1.f), 8.f * kUnitRoundoff * core);
            }
            if (pmx_valid) {
                const float mx = d.pmx[p];
                u = fminf(u, mx + fmaxf(d.perr[p], 1e-4f * (mx + 1.f)));
            }
            U[p] = u;
        }
    }
}

// U = min(U, d32 + err) over the FP32 minima of the kExK closest-core voxel pairs
__global__ void k_exact_tighten(const float4* __restrict__ res1, int64_t P, float* __restrict__ U) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
        float u = U[p];
        for (int k = 0; k < kExK; ++k) {
            const float4 r = res1[(size_t)kExK * p + k];
            if (r.x < FLT_MAX) u = fminf(u, r.x + err_bound(r.w) + 1e-5f * r.x + 1e-6f);
        }
        U[p] = u;
    }
}

// squared box gap of two voxels, as vox_dist2 computes it
__device__ __forceinline__ float box_gap2(const float4* a, const float4* b) {
    const float4 alo = a[0], ahi = a[1], blo = b[0], bhi = b[1];
    const float gx = fmaxf(fmaxf(alo.x - bhi.x, blo.x - ahi.x), 0.f);
    const float gy = fmaxf(fmaxf(alo.y - bhi.y, blo.y - ahi.y), 0.f);
    const float gz = fmaxf(fmaxf(alo.z - bhi.z, blo.z - ahi.z), 0.f);
    return gx * gx + gy * gy + gz * gz;
}

// count (WRITE = false) or write the candidate voxel pairs of every reported pair
// The preset of a candidate is U plus the largest FP32 error its minimum can
// carry: err_bound of a coordinate bound R <= gap + both voxel diagonals, as
// every coordinate is taken relative to a vertex of the A voxel.
template <bool WRITE>
__global__ void __launch_bounds__(kBlk) k_exact_vp(JoinDev d, const float* __restrict__ Ub,
                                                   const uint32_t* __restrict__ vt1,
                                                   const uint32_t* __restrict__ vt2, int64_t* __restrict__ cnt,
                                                   const int64_t* __restrict__ off, RefineItem* __restrict__ items,
                                                   int* __restrict__ item_pair, float* __restrict__ preset) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        if (d.pstat[p] != kReported) {
            if (!WRITE && lane == 0) cnt[p] = 0;
            continue;
        }
        const int q = d.pq[p], t = d.pt[p];
        const uint32_t a0 = d.ovox1[q], b0 = d.ovox2[t];
        const uint32_t n1 = d.ovox1[q + 1] - a0, n2 = d.ovox2[t + 1] - b0;
        const float U = Ub[p];
        const float lim = U * (1.f + 1e-5f) + 1e-6f;
        const float lim2 = lim * lim;
        const uint64_t total = (uint64_t)n1 * n2;
        int64_t pos = WRITE ? off[p] : 0, count = 0;
        for (uint64_t base = 0; base < total; base += 32) {
            const uint64_t k = base + lane;
            bool keep = false;
            uint32_t a = 0, b = 0;
            if (k < total) {
                a = a0 + (uint32_t)(k / n2);
                b = b0 + (uint32_t)(k % n2);
                keep = box_gap2(d.vox1 + 3 * (size_t)a, d.vox2 + 3 * (size_t)b) <= lim2 && vt1[a + 1] > vt1[a] &&
                       vt2[b + 1] > vt2[b];
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (WRITE && keep) {
                const int64_t w = pos + __popc(bal & ((1u << lane) - 1u));
                items[w] = RefineItem{vt1[a], vt1[a + 1] - vt1[a], vt2[b], vt2[b + 1] - vt2[b]};
                item_pair[w] = p;
                const float4* va = d.vox1 + 3 * (size_t)a;
                const float4* vb = d.vox2 + 3 * (size_t)b;
                const float4 alo = va[0], ahi = va[1], blo = vb[0], bhi = vb[1];
                const float da = (ahi.x - alo.x) + (ahi.y - alo.y) + (ahi.z - alo.z);
                const float db = (bhi.x - blo.x) + (bhi.y - blo.y) + (bhi.z - blo.z);
                const float R = (U + da + db) * 1.001f + 1.f;
                preset[w] = U + 2.f * err_bound(R) + 1e-6f;
            }
            pos += __popc(bal);
            count += __popc(bal);
        }
        if (!WRITE && lane == 0) cnt[p] = count;
    }
}

constexpr int kRjWarps = 8;
constexpr int kRjCA = 128;  // A triangles staged per round, as the refine stages them

// The FP32 pass's item-level test on its own, ahead of the refine: a small
// kernel (no queue, no triangle distances) that keeps the candidates which
// may have a triangle pair below their preset and compacts them -- item,
// object pair, preset -- for the refine.  About 92 % of the candidates of
// the within-400 join fall here; in the refine the same test shared a large
// kernel's instruction cache and registers with the evaluations.
__global__ void __launch_bounds__(kRjWarps * 32) k_exact_reject(const float4* __restrict__ triA,
                                                                const float4* __restrict__ triB,
                                                                const RefineItem* __restrict__ items,
                                                                const int* __restrict__ item_pair,
                                                                const float* __restrict__ preset, int64_t E,
                                                                RefineItem* __restrict__ out_items,
                                                                int* __restrict__ out_pair,
                                                                float* __restrict__ out_preset,
                                                                unsigned* __restrict__ n_out) {
    __shared__ __align__(16) float4 stage[kRjWarps][2 * kRjCA + 2 * (kRjCA / kCl)];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float4* sphA = stage[wid];
    float4* auxA = sphA + kRjCA;
    float4* clS = auxA + kRjCA;
    float4* clA = clS + kRjCA / kCl;
    // each warp takes a contiguous run of candidates: those of one object
    // pair come A voxel by A voxel, so consecutive candidates mostly share
    // their A voxel, whose staging (and the axis it was staged along) is
    // then reused -- any axis gives a valid bound
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t per = (E + nw - 1) / nw;
    const int64_t e_end = min(E, (gw + 1) * per);
    uint32_t held_off = 0, held_cnt = 0;  // the A voxel staged (held_cnt 0: none)
    float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float3 u = make_float3(0.f, 0.f, 0.f);
    ChunkBound vb{};
    for (int64_t e = gw * per; e < e_end; ++e) {
        const RefineItem it = items[e];
        if (it.a_cnt == 0 || it.b_cnt == 0) continue;  // nothing to refine
        const float bd = preset[e];
        bool keep;
        if (it.a_cnt <= (uint32_t)kRjCA) {
            if (it.a_off != held_off || it.a_cnt != held_cnt) {
                o4 = triA[(size_t)it.a_off * kTriF4];
                const float4 q = triB[(size_t)it.b_off * kTriF4];  // first A vertex to first B vertex
                const float ux = q.x - o4.x, uy = q.y - o4.y, uz = q.z - o4.z;
                const float n2 = ux * ux + uy * uy + uz * uz;
                const float inv = n2 > 0.f ? rsqrtf(n2) : 0.f;
                u = make_float3(ux * inv, uy * inv, uz * inv);
                vb = stage_a_chunk<kRjCA, true>(triA, it, 0, (int)it.a_cnt, o4, u, sphA, auxA, clS, clA, lane);
                held_off = it.a_off;
                held_cnt = it.a_cnt;
            }
            keep = b_needs_chunk<true>(triB, it, ((int)it.a_cnt + kCl - 1) / kCl, vb, o4, u, bd, clS, clA, lane);
        } else {  // a voxel larger than one staging round
            const float4 oa = triA[(size_t)it.a_off * kTriF4];
            const float4 q = triB[(size_t)it.b_off * kTriF4];
            const float ux = q.x - oa.x, uy = q.y - oa.y, uz = q.z - oa.z;
            const float n2 = ux * ux + uy * uy + uz * uz;
            const float inv = n2 > 0.f ? rsqrtf(n2) : 0.f;
            const float3 ua = make_float3(ux * inv, uy * inv, uz * inv);
            keep = item_may_go_below<kRjCA, true>(triA, triB, it, oa, ua, bd, sphA, auxA, clS, clA, lane);
            held_cnt = 0;  // the staging was overwritten
        }
        if (keep && lane == 0) {
            const unsigned w = atomicAdd(n_out, 1u);
            out_items[w] = it;
            out_pair[w] = item_pair[e];
            out_preset[w] = bd;
        }
    }
}

// per object pair: best32 = min d32, emax = max error bound (non-negative
// floats order like their bit patterns)
// counts[0]: items the refine's item-level test dropped (rmax 0, nothing
// staged); counts[1]: items with a triangle pair below their preset
__global__ void k_exact_best(const float4* __restrict__ res, const int* __restrict__ item_pair, int64_t E,
                             unsigned* __restrict__ best32, unsigned* __restrict__ emax,
                             unsigned* __restrict__ counts) {
    unsigned dropped = 0, below = 0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const float4 r = res[e];
        if (!(r.x < FLT_MAX)) {  // no triangle pair below the preset
            dropped += r.w == 0.f;
            continue;
        }
        ++below;
        const int p = item_pair[e];
        atomicMin(best32 + p, __float_as_uint(fmaxf(r.x, 0.f)));
        atomicMax(emax + p, __float_as_uint(err_bound(r.w)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dropped += __shfl_xor_sync(0xffffffffu, dropped, o);
        below += __shfl_xor_sync(0xffffffffu, below, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (dropped) atomicAdd(counts, dropped);
        if (below) atomicAdd(counts + 1, below);
    }
}

// candidates that can still hold the minimum, compacted (order is irrelevant)
__global__ void k_exact_select(const float4* __restrict__ res, const RefineItem* __restrict__ items,
                               const int* __restrict__ item_pair, int64_t E, const unsigned* __restrict__ best32,
                               const unsigned* __restrict__ emax, RefineItem* __restrict__ sel,
                               int* __restrict__ sel_pair, float2* __restrict__ sel_thr, unsigned* __restrict__ n_sel) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const float x = res[e].x;
        if (!(x < FLT_MAX)) continue;
        const int p = item_pair[e];
        const float b = __uint_as_float(best32[p]), m = __uint_as_float(emax[p]);
        if (x - m <= b + m) {
            const unsigned w = atomicAdd(n_sel, 1u);
            sel[w] = items[e];
            sel_pair[w] = p;
            sel_thr[w] = make_float2(b + 2.f * m, b + m);  // sphere reach, FP64 limit
        }
    }
}

__device__ __forceinline__ void sphere_rel(const float4* t, float4 o, float& cx, float& cy, float& cz, float& r) {
    const float4 v0 = t[0], v1 = t[1], v2 = t[2];
    const float x0 = v0.x - o.x, y0 = v0.y - o.y, z0 = v0.z - o.z;
    const float x1 = v1.x - o.x, y1 = v1.y - o.y, z1 = v1.z - o.z;
    const float x2 = v2.x - o.x, y2 = v2.y - o.y, z2 = v2.z - o.z;
    cx = (x0 + x1 + x2) * (1.f / 3.f);
    cy = (y0 + y1 + y2) * (1.f / 3.f);
    cz = (z0 + z1 + z2) * (1.f / 3.f);
    float r2 = (x0 - cx) * (x0 - cx) + (y0 - cy) * (y0 - cy) + (z0 - cz) * (z0 - cz);
    r2 = fmaxf(r2, (x1 - cx) * (x1 - cx) + (y1 - cy) * (y1 - cy) + (z1 - cz) * (z1 - cz));
    r2 = fmaxf(r2, (x2 - cx) * (x2 - cx) + (y2 - cy) * (y2 - cy) + (z2 - cz) * (z2 - cz));
    // inflated so FP32 rounding never drops a pair that could be the minimum
    r = radius_sqrt(r2) * 1.0001f + 1e-5f * (fabsf(cx) + fabsf(cy) + fabsf(cz)) + 1e-6f;
}

// extent of a triangle's projection on the unit axis u, relative to o,
// widened like the refine's staged bounds
__device__ __forceinline__ float2 proj_rel(const float4* t, float4 o, float3 u) {
    const float4 a = t[0], b = t[1], c = t[2];
    const float p0 = (a.x - o.x) * u.x + (a.y - o.y) * u.y + (a.z - o.z) * u.z;
    const float p1 = (b.x - o.x) * u.x + (b.y - o.y) * u.y + (b.z - o.z) * u.z;
    const float p2 = (c.x - o.x) * u.x + (c.y - o.y) * u.y + (c.z - o.z) * u.z;
    const float mg = 1e-5f * (fabsf(p0) + fabsf(p1) + fabsf(p2)) + 1e-6f;
    return make_float2(fminf(p0, fminf(p1, p2)) - mg, fmaxf(p0, fmaxf(p1, p2)) + mg);
}

__device__ __forceinline__ void pre64(const float4* t, double ox, double oy, double oz, PreTri<double>& P) {
    const float4 a = t[0], b = t[1], c = t[2];
    pretri(P, v3<double>(a.x - ox, a.y - oy, a.z - oz), v3<double>(b.x - ox, b.y - oy, b.z - oz),
           v3<double>(c.x - ox, c.y - oy, c.z - oz));
}

// the FP32 operands as the refine forms them (translated to o), and the
// largest |coordinate| after translation (the R of the error model)
__device__ __forceinline__ float pre32(const float4* t, float4 o, PreTri<float>& P) {
    const float4 a = t[0], b = t[1], c = t[2];
    const V3<float> x = v3<float>(a.x - o.x, a.y - o.y, a.z - o.z), y = v3<float>(b.x - o.x, b.y - o.y, b.z - o.z),
                    z = v3<float>(c.x - o.x, c.y - o.y, c.z - o.z);
    pretri(P, x, y, z);
    float r = 0.f;
    r = fmaxf(r, fmaxf(fabsf(x.x), fmaxf(fabsf(x.y), fabsf(x.z))));
    r = fmaxf(r, fmaxf(fabsf(y.x), fmaxf(fabsf(y.y), fabsf(y.z))));
    return fmaxf(r, fmaxf(fabsf(z.x), fmaxf(fabsf(z.y), fabsf(z.z))));
}

constexpr int kExWarps = 4;
constexpr int kExQueue = 64;  // queued triangle pairs per warp (>= 32 + 31)

// FP32 distance with its error bound, and the FP64 distance when the pair can
// still be the minimum (d32 - e <= lim), of triangle pair (a, b) of an item
__device__ __forceinline__ double exact_pair(const float4* ta, const float4* tb, float4 o4, float lim) {
    PreTri<float> A32, B32;
    const float rA = pre32(ta, o4, A32);
    const float rB = pre32(tb, o4, B32);
    const float d32 = sqrtf(tri_dist2(A32, B32));
    if (d32 - err_bound(fmaxf(rA, rB)) > lim) return 1e300;
    PreTri<double> A, B;
    const double ox = o4.x, oy = o4.y, oz = o4.z;
    pre64(ta, ox, oy, oz, A);
    pre64(tb, ox, oy, oz, B);
    return tri_dist2(A, B);
}

// FP64 minimum over the triangle pairs of a selected voxel pair whose FP32
// bounding-sphere gap and cylinder bound (cyl_keep, along the axis from the
// item's first A vertex to its first B vertex) are <= the item's reach and
// whose FP32 distance, less its
// error bound, is <= the item's limit; one warp per item.  Lane j owns B
// triangle j of the current chunk of 32 and tests it against the A chunk's
// spheres (staged in shared memory); the pairs that pass are queued, and
// every 32 queued pairs are evaluated one per lane, so the evaluations run
// with the whole warp instead of with the few lanes whose test passed.
__global__ void __launch_bounds__(kExWarps * 32) k_exact_f64(const float4* __restrict__ triA,
                                                             const float4* __restrict__ triB,
                                                             const RefineItem* __restrict__ sel,
                                                             const int* __restrict__ sel_pair,
                                                             const float2* __restrict__ sel_thr,
                                                             const unsigned* __restrict__ n_sel,
                                                             unsigned long long* __restrict__ pexact_bits) {
    __shared__ float4 sphA[kExWarps][32];
    __shared__ float2 prjA[kExWarps][32];
    __shared__ uint2 queue[kExWarps][kExQueue];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const unsigned n = *n_sel;
    uint2* q = queue[w];
    for (unsigned it = blockIdx.x * kExWarps + w; it < n; it += gridDim.x * kExWarps) {
        const RefineItem r = sel[it];
        const float2 tl = sel_thr[it];
        const float thr = tl.x, lim = tl.y;
        const float4 o4 = triA[(size_t)r.a_off * kTriF4];
        const float4* tA = triA + (size_t)r.a_off * kTriF4;
        const float4* tB = triB + (size_t)r.b_off * kTriF4;
        // the item's axis: from the first A vertex to the first B vertex
        float3 u;
        {
            const float4 q = tB[0];
            const float ux = q.x - o4.x, uy = q.y - o4.y, uz = q.z - o4.z;
            const float n2 = ux * ux + uy * uy + uz * uz;
            const float inv = n2 > 0.f ? rsqrtf(n2) : 0.f;
            u = make_float3(ux * inv, uy * inv, uz * inv);
        }
        double best = 1e300;
        int qn = 0;
        // evaluate the first `take` queued pairs, one per lane, and move the
        // rest to the front
        auto drain = [&](int take) {
            __syncwarp();
            if (lane < take) {
                const uint2 e = q[lane];
                const double d2 = exact_pair(tA + (size_t)e.x * kTriF4, tB + (size_t)e.y * kTriF4, o4, lim);
                best = d2 < best ? d2 : best;
            }
            const uint2 moved = lane + take < qn ? q[lane + take] : make_uint2(0u, 0u);
            __syncwarp();
            if (lane + take < qn) q[lane] = moved;
            qn -= take;
            __syncwarp();
        };
        for (uint32_t b0 = 0; b0 < r.b_cnt; b0 += 32) {
            const bool bv = b0 + lane < r.b_cnt;
            float bx = 0.f, by = 0.f, bz = 0.f, br = 0.f;
            float2 pb = make_float2(0.f, 0.f);
            if (bv) {
                sphere_rel(tB + (size_t)(b0 + lane) * kTriF4, o4, bx, by, bz, br);
                pb = proj_rel(tB + (size_t)(b0 + lane) * kTriF4, o4, u);
            }
            for (uint32_t a0 = 0; a0 < r.a_cnt; a0 += 32) {
                const int ca = (int)min(32u, r.a_cnt - a0);
                __syncwarp();
                if (lane < ca) {
                    float cx, cy, cz, rr;
                    sphere_rel(tA + (size_t)(a0 + lane) * kTriF4, o4, cx, cy, cz, rr);
                    sphA[w][lane] = make_float4(cx, cy, cz, rr);
                    prjA[w][lane] = proj_rel(tA + (size_t)(a0 + lane) * kTriF4, o4, u);
                }
                __syncwarp();
                for (int i = 0; i < ca; ++i) {
                    const float4 sa = sphA[w][i];
                    const float2 pa = prjA[w][i];
                    const float dx = sa.x - bx, dy = sa.y - by, dz = sa.z - bz;
                    const float reach = sa.w + br + thr;
                    const bool keep = bv && dx * dx + dy * dy + dz * dz <= reach * reach &&
                                      cyl_keep(dx, dy, dz, sa.w + br, fmaxf(pb.x - pa.y, pa.x - pb.y), u, thr);
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if (keep) q[qn + __popc(m & lt)] = make_uint2(a0 + (uint32_t)i, b0 + (uint32_t)lane);
                    qn += __popc(m);
                    if (qn >= 32) drain(32);
                }
            }
        }
        if (qn > 0) drain(qn);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double v = __shfl_xor_sync(0xffffffffu, best, o);
            best = v < best ? v : best;
        }
        // non-negative doubles order like their bit patterns
        if (lane == 0 && best < 1e300)
            atomicMin(pexact_bits + sel_pair[it], (unsigned long long)__double_as_longlong(sqrt(best)));
    }
}

// largest |best32 - D| / max(D, 1) over the reported pairs: the FP32 refine's
// error against FP64 on this join
__global__ void k_exact_err(JoinDev d, const unsigned* __restrict__ best32, const double* __restrict__ pexact,
                            unsigned* __restrict__ err_bits) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.P; p += gridDim.x * blockDim.x) {
        if (d.pstat[p] != kReported) continue;
        const double D = pexact[p];
        if (!(D < 1e300)) continue;
        const double b = (double)__uint_as_float(best32[p]);
        const float rel = (float)(fabs(b - D) / fmax(D, 1.0));
        atomicMax(err_bits, __float_as_uint(rel));
    }
}

int grid(int64_t n, int per_block, int cap) {
    int64_t g = (n + per_block - 1) / per_block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

}  // namespace

int exact_distances(tdp_ctx* ctx, const JoinDev& d, const tdp_tile* t1, const tdp_tile* t2, bool pmx_valid,
                    double* pexact, ExactInfo& info, const LazyTile& lz1, const LazyTile& lz2) {
    cudaStream_t s = ctx->stream;
    info = ExactInfo{};
    int rc;
#define CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)
#define ENS(slot, bytes) do { if ((rc = ensure(ctx, ctx->scratch[slot], (bytes)))) return rc; } while (0)
    const size_t Pz = (size_t)std::max<int64_t>(d.P, 1);
    // every byte 0x7f: the double 1.38e306, above any distance, so atomicMin
    // over the bit patterns of non-negative doubles takes the first real value
    CU(cudaMemsetAsync(pexact, 0x7f, Pz * 8, s));
    if (d.P <= 0) return TDP_OK;
    ENS(64, (Pz + 1) * 8);             // counts
    ENS(65, (Pz + 1) * 8);             // offsets
    ENS(78, Pz * 4);                   // U per pair
    ENS(79, Pz * kExK * sizeof(RefineItem));  // phase-1 items, kExK per pair
    ENS(80, Pz * kExK * sizeof(float4));      // phase-1 FP32 results
    ENS(75, 64);                       // counters
    int64_t* cnt = (int64_t*)ctx->scratch[64].p;
    int64_t* off = (int64_t*)ctx->scratch[65].p;
    float* Ub = (float*)ctx->scratch[78].p;
    RefineItem* item1 = (RefineItem*)ctx->scratch[79].p;
    float4* res1 = (float4*)ctx->scratch[80].p;
    unsigned* ctr = (unsigned*)ctx->scratch[75].p;
    const uint32_t* vt1 = t1->vtri[kNumLods - 1];
    const uint32_t* vt2 = t2->vtri[kNumLods - 1];
    const int pg = grid(d.P, kBlk / 32, ctx->num_sms * 32);
    CU(cudaMemsetAsync(cnt + d.P, 0, 8, s));
    CU(cudaMemsetAsync(ctr, 0, 64, s));
    CU(cudaEventRecord(ctx->xev[0], s));
    k_exact_upper<<<pg, kBlk, 0, s>>>(d, pmx_valid ? 1 : 0, vt1, vt2, Ub, item1);
    CU(cudaGetLastError());
    // phase 1: the kExK closest-core voxel pairs of every object pair in FP32 tighten U
    const int64_t n1 = d.P * kExK;
    if (n1 >= (1LL << 31)) return fail(ctx, TDP_ERR_ARG, "too many object pairs for the exact-distance stage");
    CU(launch_fetch_items(item1, nullptr, n1, kNumLods - 1, lz1, lz2, ctx->num_sms, s));
    CU(launch_refine_tuned(t1->tri[kNumLods - 1], t2->tri[kNumLods - 1], item1, (int)n1, res1, ctr, nullptr,
                           ctx->num_sms, kExactRefineCfg, s));
    k_exact_tighten<<<grid(d.P, 256, ctx->num_sms * 8), 256, 0, s>>>(res1, d.P, Ub);
    CU(cudaGetLastError());
    CU(cudaEventRecord(ctx->xev[1], s));
    k_exact_vp<false><<<pg, kBlk, 0, s>>>(d, Ub, vt1, vt2, cnt, nullptr, nullptr, nullptr, nullptr);
    CU(cudaGetLastError());
    size_t tb = 0;
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)d.P + 1, s));
    ENS(66, tb + 16);
    CU(cub::DeviceScan::ExclusiveSum(ctx->scratch[66].p, tb, cnt, off, (int)d.P + 1, s));
    int64_t E = 0;
    CU(cudaMemcpyAsync(&E, off + d.P, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    info.launches += 6 + (lz1.on || lz2.on ? 1 : 0);
    info.items = (long)E;
    if (E >= (1LL << 31)) return fail(ctx, TDP_ERR_ARG, "too many voxel pairs for the exact-distance stage");
    const size_t Ez = (size_t)std::max<int64_t>(E, 1);
    ENS(67, Ez * sizeof(RefineItem));  // items
    ENS(68, Ez * 4);                   // item -> pair
    ENS(69, Ez * sizeof(float4));      // FP32 results
    ENS(70, Pz * 4);                   // best32
    ENS(71, Pz * 4);                   // emax
    ENS(72, Ez * sizeof(RefineItem));  // selected items
    ENS(73, Ez * 4);                   // selected -> pair
    ENS(74, Ez * 8);                   // selected (reach, limit)
    ENS(81, Ez * 4);                   // presets
    ENS(84, Ez * sizeof(RefineItem));  // items that pass the item-level test
    ENS(85, Ez * 4);                   // their pairs
    ENS(86, Ez * 4);                   // their presets
    RefineItem* items = (RefineItem*)ctx->scratch[67].p;
    int* item_pair = (int*)ctx->scratch[68].p;
    float4* res = (float4*)ctx->scratch[69].p;
    unsigned* best32 = (unsigned*)ctx->scratch[70].p;
    unsigned* emax = (unsigned*)ctx->scratch[71].p;
    RefineItem* sel = (RefineItem*)ctx->scratch[72].p;
    int* sel_pair = (int*)ctx->scratch[73].p;
    float2* sel_thr = (float2*)ctx->scratch[74].p;
    float* preset = (float*)ctx->scratch[81].p;
    ctr = (unsigned*)ctx->scratch[75].p;
    k_exact_vp<true><<<pg, kBlk, 0, s>>>(d, Ub, vt1, vt2, nullptr, off, items, item_pair, preset);
    CU(cudaGetLastError());
    CU(cudaMemsetAsync(best32, 0x7f, Pz * 4, s));  // 0x7f7f7f7f = 3.4e38, above any distance
    CU(cudaMemsetAsync(emax, 0, Pz * 4, s));
    CU(cudaMemsetAsync(ctr, 0, 64, s));
    CU(cudaEventRecord(ctx->xev[2], s));
    // ctr: [0] work counter, [4] selected items, [8] FP32 error bits, [12..13] full evaluations (u64),
    // [14] items the item-level test dropped, [15] items below their preset
    unsigned long long* n_full = reinterpret_cast<unsigned long long*>(ctr + 12);
    if (E > 0) {
        CU(launch_fetch_items(items, nullptr, E, kNumLods - 1, lz1, lz2, ctx->num_sms, s));
        // the item-level test first, in its own kernel; ctr[2] counts the survivors
        RefineItem* items2 = (RefineItem*)ctx->scratch[84].p;
        int* pair2 = (int*)ctx->scratch[85].p;
        float* preset2 = (float*)ctx->scratch[86].p;
        k_exact_reject<<<grid(E, kRjWarps, ctx->num_sms * 16), kRjWarps * 32, 0, s>>>(
            t1->tri[kNumLods - 1], t2->tri[kNumLods - 1], items, item_pair, preset, E, items2, pair2, preset2, ctr + 2);
        CU(cudaGetLastError());
        unsigned e2 = 0;
        CU(cudaMemcpyAsync(&e2, ctr + 2, 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        const int64_t E2 = e2;
        info.launches += 1;
        if (E2 > 0)
            CU(launch_refine_tuned(t1->tri[kNumLods - 1], t2->tri[kNumLods - 1], items2, (int)E2, res, ctr, n_full,
                                   ctx->num_sms, kExactRefineCfg, s, nullptr, preset2));
        const int eg = grid(std::max<int64_t>(E2, 1), 256, ctx->num_sms * 16);
        k_exact_best<<<eg, 256, 0, s>>>(res, pair2, E2, best32, emax, ctr + 14);
        CU(cudaGetLastError());
        k_exact_select<<<eg, 256, 0, s>>>(res, items2, pair2, E2, best32, emax, sel, sel_pair, sel_thr, ctr + 4);
        CU(cudaGetLastError());
        CU(cudaEventRecord(ctx->xev[3], s));
        k_exact_f64<<<ctx->num_sms * 8, kExWarps * 32, 0, s>>>(t1->tri[kNumLods - 1], t2->tri[kNumLods - 1], sel,
                                                              sel_pair, sel_thr, ctr + 4,
                                                              reinterpret_cast<unsigned long long*>(pexact));
        CU(cudaGetLastError());
        k_exact_err<<<grid(d.P, 256, ctx->num_sms * 8), 256, 0, s>>>(d, best32, pexact, ctr + 8);
        CU(cudaGetLastError());
        CU(cudaEventRecord(ctx->xev[4], s));
        info.launches += 6 + (lz1.on || lz2.on ? 1 : 0);
        unsigned ns[12] = {0};
        CU(cudaMemcpyAsync(ns, ctr + 4, 48, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        info.f64_items = ns[0];
        float e32;
        std::memcpy(&e32, &ns[4], 4);
        info.max_rel_err32 = e32;
        std::memcpy(&info.full_evals, &ns[8], 8);
        info.dropped_items = (long)(E - E2) + ns[10];
        info.below_items = ns[11];
        float ms[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], ctx->xev[k], ctx->xev[k + 1]);
        for (int k = 0; k < 4; ++k) info.phase_ms[k] = ms[k];
    }
#undef ENS
#undef CU
    return TDP_OK;
}

}  // namespace tdp
