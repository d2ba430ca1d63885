// refine.cu -- the LOD refine: for every voxel pair, the minimum triangle
// distance and the two Hausdorff-widened bounds over all triangle pairs.
//
// Reference: TriDist_cuda_op_shm_flat_fused (src/geometry/computing_gpu.cu:1069-1152),
// launched one CTA of 512 threads per voxel pair by
// MeshDist_batch_gpu_op_shm_flat_stream (computing_gpu.cu:6540-6658).
// Outputs per voxel pair (float4):
//   x = min d,  y = min max(d - ph1 - ph2, 0),  z = min d + h1 + h2,
//   w = R, the largest |coordinate| after translation to the pair origin
//       (the FP32 error bound of x is err_bound(R), see common.cuh).
//
// Two forms:
//   refine_plain_kernel  one CTA per voxel pair, both voxels staged in shared
//                        memory, every triangle pair fully evaluated.  This is the
//                        "plain GPU form" the tuned form is measured against.
//   refine_tuned_kernel  persistent, one warp per voxel pair pulled from an atomic
//                        work counter; triangles are pre-processed once into
//                        shared memory, each lane owns one B-side triangle, and
//                        cluster- then triangle-level lower bounds against the
//                        warp's running minima skip pairs that cannot lower any
//                        of the three minima (details above the kernel).
#include <float.h>
#include "common.cuh"
#include "tridist.cuh"
#include "cull.cuh"
#include "refine.cuh"

namespace tdp {

__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ------------------------------------------------------------------ plain form
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) refine_plain_kernel(const float4* __restrict__ triA,
                                                             const float4* __restrict__ triB,
                                                             const RefineItem* __restrict__ items,
                                                             int n_items, float4* __restrict__ out) {
    constexpr int CH = 128;  // triangles staged per side per round
    __shared__ float4 sa[CH * kTriF4];
    __shared__ float4 sb[CH * kTriF4];
    __shared__ float red[4][BLOCK / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RefineItem w = items[it];
        if (w.a_cnt == 0 || w.b_cnt == 0) {
            if (tid == 0) out[it] = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
            continue;
        }
        const float4 o4 = triA[(size_t)w.a_off * kTriF4];
        float dmin = FLT_MAX, lomin = FLT_MAX, himin = FLT_MAX, rmax = 0.f;
        for (uint32_t a0 = 0; a0 < w.a_cnt; a0 += CH) {
            const int ca = min((uint32_t)CH, w.a_cnt - a0);
            for (uint32_t b0 = 0; b0 < w.b_cnt; b0 += CH) {
                const int cb = min((uint32_t)CH, w.b_cnt - b0);
                __syncthreads();
                for (int k = tid; k < ca * kTriF4; k += BLOCK) {
                    float4 t = triA[((size_t)w.a_off + a0) * kTriF4 + k];
                    t.x -= o4.x; t.y -= o4.y; t.z -= o4.z;
                    rmax = fmaxf(rmax, fmaxf(fabsf(t.x), fmaxf(fabsf(t.y), fabsf(t.z))));
                    sa[k] = t;
                }
                for (int k = tid; k < cb * kTriF4; k += BLOCK) {
                    float4 t = triB[((size_t)w.b_off + b0) * kTriF4 + k];
                    t.x -= o4.x; t.y -= o4.y; t.z -= o4.z;
                    rmax = fmaxf(rmax, fmaxf(fabsf(t.x), fmaxf(fabsf(t.y), fabsf(t.z))));
                    sb[k] = t;
                }
                __syncthreads();
                for (int p = tid; p < ca * cb; p += BLOCK) {
                    const int i = p / cb, j = p - i * cb;
                    const float4 a0v = sa[3 * i], a1v = sa[3 * i + 1], a2v = sa[3 * i + 2];
                    const float4 b0v = sb[3 * j], b1v = sb[3 * j + 1], b2v = sb[3 * j + 2];
                    PreTri<float> A, B;
                    pretri(A, v3(a0v.x, a0v.y, a0v.z), v3(a1v.x, a1v.y, a1v.z), v3(a2v.x, a2v.y, a2v.z));
                    pretri(B, v3(b0v.x, b0v.y, b0v.z), v3(b1v.x, b1v.y, b1v.z), v3(b2v.x, b2v.y, b2v.z));
                    const float d = sqrtf(tri_dist2(A, B));
                    dmin = fminf(dmin, d);
                    lomin = fminf(lomin, fmaxf(d - a0v.w - b0v.w, 0.f));
                    himin = fminf(himin, d + a1v.w + b1v.w);
                }
            }
        }
        dmin = warp_min(dmin); lomin = warp_min(lomin); himin = warp_min(himin); rmax = warp_max(rmax);
        __syncthreads();
        if (lane == 0) { red[0][wid] = dmin; red[1][wid] = lomin; red[2][wid] = himin; red[3][wid] = rmax; }
        __syncthreads();
        if (tid == 0) {
            for (int k = 1; k < BLOCK / 32; ++k) {
                dmin = fminf(dmin, red[0][k]); lomin = fminf(lomin, red[1][k]);
                himin = fminf(himin, red[2][k]); rmax = fmaxf(rmax, red[3][k]);
            }
            out[it] = make_float4(dmin, lomin, himin, rmax);
        }
    }
}

// ------------------------------------------------------------------ tuned form
// One warp per voxel pair, pulled from an atomic work counter by a persistent
// grid (the next index is claimed while the current pair is processed).  Per
// chunk of up to 64 A-side triangles, staged once, and per chunk of 32 B-side
// triangles (one per lane):
//   1. both sides are pre-processed once into shared memory (structure of
//      arrays: a broadcast read of one triangle by the whole warp is one
//      transaction per field); each triangle also gets a bounding sphere
//      (cx, cy, cz, r) and (ph, h, axis projection) as two float4 records;
//   2. the A chunk is cut into clusters of 8 consecutive triangles (a voxel's
//      triangles are stored in mesh order, so consecutive triangles are
//      close); a cluster carries a sphere holding its members' spheres, its
//      largest axis projection, its largest ph and smallest h;
//   3. seed: lane j picks the cluster, then the member, whose bound is nearest
//      its B triangle j and evaluates that pair fully, so the three running
//      minima start close to their final values;
//   4. cull: for every cluster (warp-uniform loop) lane j tests the cluster's
//      lower bounds against the minima; a cluster no lane needs is skipped
//      whole, otherwise its members are tested one by one with the same two
//      bounds -- the bounding-sphere gap and the gap between the triangles'
//      projections on the axis u joining the two voxels (projection onto a
//      unit vector never increases a distance) -- and pairs that could still
//      lower a minimum are appended to a shared-memory queue with a warp ballot;
//   5. drain: whenever 32 pairs are queued, each lane evaluates one of them
//      fully, so the expensive test never runs with idle lanes.
// A pair is skipped only when a lower bound of d(i, j) is >= max(best_d,
// best_lo + phA + phB, best_hi - hA - hB), so it can lower none of the minima;
// a cluster only when its bound is >= that threshold taken with the cluster's
// largest ph and smallest h, which is >= every member's threshold.
constexpr int kPreF = 37;   // PreTri floats, structure of arrays
constexpr int kQueue = 64;  // queued pairs per warp (>= 32 + 31)

// Per-warp shared memory of the tuned kernel for CA A-side triangles per
// chunk, in floats (every float4 array starts 16-byte aligned).
template <int CA>
struct TunedLayout {
    static_assert(CA % kCl == 0 && CA <= 256, "A chunk must be whole clusters and fit the queue's 8-bit index");
    static constexpr int kNCl = CA / kCl;
    static constexpr int kOffSphA = kPreF * CA;
    static constexpr int kOffAuxA = kOffSphA + 4 * CA;
    static constexpr int kOffClS = kOffAuxA + 4 * CA;
    static constexpr int kOffClA = kOffClS + 4 * kNCl;
    static constexpr int kOffPreB = kOffClA + 4 * kNCl;
    static constexpr int kOffAuxB = kOffPreB + kPreF * kCB;
    static constexpr int kOffQueue = kOffAuxB + 4 * kCB;
    static constexpr int kWarpFloats = kOffQueue + kQueue / 2;
    static_assert(kOffSphA % 4 == 0 && kOffPreB % 4 == 0 && kOffAuxB % 4 == 0 && kWarpFloats % 4 == 0,
                  "float4 arrays must stay 16-byte aligned");
};

__device__ __forceinline__ void store_pre(float* s, int ld, int k, const PreTri<float>& t) {
    float* p = s + k;
#define PUT(i, v) p[(i) * ld] = (v)
    PUT(0, t.v[0].x); PUT(1, t.v[0].y); PUT(2, t.v[0].z);
    PUT(3, t.v[1].x); PUT(4, t.v[1].y); PUT(5, t.v[1].z);
    PUT(6, t.v[2].x); PUT(7, t.v[2].y); PUT(8, t.v[2].z);
    PUT(9, t.e[0].x); PUT(10, t.e[0].y); PUT(11, t.e[0].z);
    PUT(12, t.e[1].x); PUT(13, t.e[1].y); PUT(14, t.e[1].z);
    PUT(15, t.e[2].x); PUT(16, t.e[2].y); PUT(17, t.e[2].z);
    PUT(18, t.n.x); PUT(19, t.n.y); PUT(20, t.n.z); PUT(21, t.inn);
    PUT(22, t.ee[0]); PUT(23, t.ee[1]); PUT(24, t.ee[2]);
    PUT(25, t.iee[0]); PUT(26, t.iee[1]); PUT(27, t.iee[2]);
    PUT(28, t.m[0].x); PUT(29, t.m[0].y); PUT(30, t.m[0].z);
    PUT(31, t.m[1].x); PUT(32, t.m[1].y); PUT(33, t.m[1].z);
    PUT(34, t.m[2].x); PUT(35, t.m[2].y); PUT(36, t.m[2].z);
#undef PUT
}

__device__ __forceinline__ void load_pre(const float* s, int ld, int k, PreTri<float>& t) {
    const float* p = s + k;
#define GET(i) p[(i) * ld]
    t.v[0] = v3(GET(0), GET(1), GET(2)); t.v[1] = v3(GET(3), GET(4), GET(5)); t.v[2] = v3(GET(6), GET(7), GET(8));
    t.e[0] = v3(GET(9), GET(10), GET(11)); t.e[1] = v3(GET(12), GET(13), GET(14)); t.e[2] = v3(GET(15), GET(16), GET(17));
    t.n = v3(GET(18), GET(19), GET(20)); t.inn = GET(21);
    t.ee[0] = GET(22); t.ee[1] = GET(23); t.ee[2] = GET(24);
    t.iee[0] = GET(25); t.iee[1] = GET(26); t.iee[2] = GET(27);
    t.m[0] = v3(GET(28), GET(29), GET(30)); t.m[1] = v3(GET(31), GET(32), GET(33)); t.m[2] = v3(GET(34), GET(35), GET(36));
#undef GET
}

__device__ __forceinline__ void tri_sphere(const PreTri<float>& t, float3& c, float& r) {
    c = make_float3((t.v[0].x + t.v[1].x + t.v[2].x) * (1.f / 3.f), (t.v[0].y + t.v[1].y + t.v[2].y) * (1.f / 3.f),
                    (t.v[0].z + t.v[1].z + t.v[2].z) * (1.f / 3.f));
    float r2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float dx = t.v[k].x - c.x, dy = t.v[k].y - c.y, dz = t.v[k].z - c.z;
        r2 = fmaxf(r2, dx * dx + dy * dy + dz * dz);
    }
    // inflate so FP32 rounding of the centre/radius can never cull a needed pair
    r = radius_sqrt(r2) * 1.0001f + 1e-6f;
}

// Stage triangle record `idx`: its PreTri fields into column k of a structure
// of arrays (leading dimension ld); returns sphere = (centre, radius) and
// aux = (ph, h, projection on u).  The projection is the triangle's largest
// (A side, far = false) or smallest (B side, far = true) one.
__device__ __forceinline__ void stage_one(const float4* __restrict__ tri, size_t idx, float4 o, float* s, int ld,
                                          int k, float3 u, bool far, float& rmax, float4& sph, float4& aux) {
    const float4* t = tri + idx * kTriF4;
    const float4 t0 = t[0], t1 = t[1], t2 = t[2];
    PreTri<float> P;
    pretri(P, v3(t0.x - o.x, t0.y - o.y, t0.z - o.z), v3(t1.x - o.x, t1.y - o.y, t1.z - o.z),
           v3(t2.x - o.x, t2.y - o.y, t2.z - o.z));
    float3 c;
    float r;
    tri_sphere(P, c, r);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        rmax = fmaxf(rmax, fmaxf(fabsf(P.v[q].x), fmaxf(fabsf(P.v[q].y), fabsf(P.v[q].z))));
    store_pre(s, ld, k, P);
    const float p0 = P.v[0].x * u.x + P.v[0].y * u.y + P.v[0].z * u.z;
    const float p1 = P.v[1].x * u.x + P.v[1].y * u.y + P.v[1].z * u.z;
    const float p2 = P.v[2].x * u.x + P.v[2].y * u.y + P.v[2].z * u.z;
    // one ulp-scale margin keeps the bound conservative under FP32 rounding
    const float mg = 1e-5f * (fabsf(p0) + fabsf(p1) + fabsf(p2)) + 1e-6f;
    sph = make_float4(c.x, c.y, c.z, r);
    aux = make_float4(t0.w, t1.w, far ? fminf(p0, fminf(p1, p2)) - mg : fmaxf(p0, fmaxf(p1, p2)) + mg, 0.f);
}

// the three minima are >= 0, so their bit patterns order like unsigned ints
__device__ __forceinline__ float warp_min_nonneg(float v) {
    return __uint_as_float(__reduce_min_sync(0xffffffffu, __float_as_uint(v)));
}


template <int WARPS, int CA, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) refine_tuned_kernel(const float4* __restrict__ triA,
                                                                     const float4* __restrict__ triB,
                                                                     const RefineItem* __restrict__ items,
                                                                     int n_items_host, const unsigned* n_items_dev,
                                                                     float4* __restrict__ out,
                                                                     unsigned* __restrict__ work_counter,
                                                                     unsigned long long* __restrict__ n_full,
                                                                     const float* __restrict__ init_bd) {
    extern __shared__ __align__(16) float smem[];
    // the item count comes from device memory when the producer ran on the GPU
    const int n_items = n_items_dev ? (int)*n_items_dev : n_items_host;
    using L = TunedLayout<CA>;
    constexpr int kCA = CA;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* ws = smem + (size_t)wid * L::kWarpFloats;
    float* sA = ws;
    float4* sphA = reinterpret_cast<float4*>(ws + L::kOffSphA);
    float4* auxA = reinterpret_cast<float4*>(ws + L::kOffAuxA);
    float4* clS = reinterpret_cast<float4*>(ws + L::kOffClS);
    float4* clA = reinterpret_cast<float4*>(ws + L::kOffClA);
    float* sB = ws + L::kOffPreB;
    float4* auxB = reinterpret_cast<float4*>(ws + L::kOffAuxB);
    unsigned short* queue = reinterpret_cast<unsigned short*>(ws + L::kOffQueue);
    const unsigned lt_mask = (1u << lane) - 1u;
    unsigned long long full_evals = 0;

    unsigned it = 0;
    if (lane == 0) it = atomicAdd(work_counter, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    while (it < (unsigned)n_items) {
        // claim the next pair now; the atomic's latency hides behind this one
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(work_counter, 1u);
        const RefineItem w = items[it];
        if (w.a_cnt == 0 || w.b_cnt == 0) {
            if (lane == 0) out[it] = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
            it = __shfl_sync(0xffffffffu, next, 0);
            continue;
        }
        const float4 o4 = triA[(size_t)w.a_off * kTriF4];
        // separation axis: from the A voxel's first vertex to the B voxel's first vertex
        float3 u;
        {
            const float4 q = triB[(size_t)w.b_off * kTriF4];
            const float ux = q.x - o4.x, uy = q.y - o4.y, uz = q.z - o4.z;
            const float n2 = ux * ux + uy * uy + uz * uz;
            const float inv = n2 > 0.f ? rsqrtf(n2) : 0.f;
            u = make_float3(ux * inv, uy * inv, uz * inv);
        }
        float bd = FLT_MAX, bl = FLT_MAX, bh = FLT_MAX, rmax = 0.f;
        // with init_bd (the exact-distance stage, and a join's last LOD) only
        // the minimum distance matters: it starts at the item's bound, and the
        // two Hausdorff minima are parked at -FLT_MAX so they never widen a
        // threshold.  An item preset to FLT_MAX has no bound and skips the
        // item-level test.
        float b_init = FLT_MAX;
        if (init_bd) {
            b_init = init_bd[it];
            bd = b_init;
            bl = -FLT_MAX;
            bh = -FLT_MAX;
            // item-level reject before any PreTri work: bounding spheres of the
            // A triangles (clustered as below) against each lane's B triangle;
            // if no pair of spheres is closer than the preset, no triangle pair
            // is, and the item has nothing below it
            bool need = !(b_init < FLT_MAX);
            for (uint32_t a0 = 0; a0 < w.a_cnt && !__any_sync(0xffffffffu, need); a0 += kCA) {
                const int ca = min((uint32_t)kCA, w.a_cnt - a0);
                const int ncl = (ca + kCl - 1) / kCl;
                __syncwarp();
                for (int k = lane; k < ca; k += 32) {
                    sphA[k] = quick_sphere(triA + ((size_t)w.a_off + a0 + k) * kTriF4, o4);
                    auxA[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                __syncwarp();
                build_clusters<CA>(sphA, auxA, ca, clS, clA, lane);
                __syncwarp();
                for (uint32_t b0 = 0; b0 < w.b_cnt && !need; b0 += kCB) {
                    if (b0 + lane >= w.b_cnt) break;
                    const float4 sb = quick_sphere(triB + ((size_t)w.b_off + b0 + lane) * kTriF4, o4);
                    for (int c = 0; c < ncl; ++c) {
                        const float4 cs = clS[c];
                        const float dx = cs.x - sb.x, dy = cs.y - sb.y, dz = cs.z - sb.z;
                        const float reach = cs.w + sb.w + bd;
                        if (dx * dx + dy * dy + dz * dz < reach * reach) { need = true; break; }
                    }
                }
            }
            if (!__any_sync(0xffffffffu, need)) {
                if (lane == 0) out[it] = make_float4(FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
                it = __shfl_sync(0xffffffffu, next, 0);
                continue;
            }
        }
        for (uint32_t a0 = 0; a0 < w.a_cnt; a0 += kCA) {
            const int ca = min((uint32_t)kCA, w.a_cnt - a0);
            const int ncl = (ca + kCl - 1) / kCl;
            __syncwarp();
            for (int k = lane; k < ca; k += 32)
                stage_one(triA, (size_t)w.a_off + a0 + k, o4, sA, kCA, k, u, false, rmax, sphA[k], auxA[k]);
            __syncwarp();
            build_clusters<CA>(sphA, auxA, ca, clS, clA, lane);
            for (uint32_t b0 = 0; b0 < w.b_cnt; b0 += kCB) {
                const int cb = min((uint32_t)kCB, w.b_cnt - b0);
                __syncwarp();
                // B side: lane j stages triangle j and keeps its bounds in registers
                const bool bval = lane < cb;
                float4 sb = make_float4(0.f, 0.f, 0.f, 0.f), ab = make_float4(0.f, 0.f, 0.f, 0.f);
                if (bval) {
                    stage_one(triB, (size_t)w.b_off + b0 + lane, o4, sB, kCB, lane, u, true, rmax, sb, ab);
                    auxB[lane] = ab;
                }
                __syncwarp();
                // seed: the nearest cluster by its bound, then its nearest member;
                // the seeds are queued and drained before anything is culled
                int seed = -1;
                float seed_lb = FLT_MAX;
                // only while the distance minimum is still unset (the first chunk
                // pair of an item, or a preset bound): later chunk pairs start from
                // tight minima and go straight to the cull
                const bool want_seed = bd == FLT_MAX || init_bd != nullptr;
                if (bval && want_seed) {
                    float best = FLT_MAX;
                    int bc = 0;
                    for (int c = 0; c < ncl; ++c) {
                        const float4 s = clS[c];
                        const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                        const float lb = fmaxf(approx_len(dx * dx + dy * dy + dz * dz) - s.w - sb.w, ab.z - clA[c].z);
                        if (lb < best) { best = lb; bc = c; }
                    }
                    best = FLT_MAX;
                    const int mend = min(ca, (bc + 1) * kCl);
                    for (int i = bc * kCl; i < mend; ++i) {
                        const float4 s = sphA[i];
                        const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                        const float lb = fmaxf(approx_len(dx * dx + dy * dy + dz * dz) - s.w - sb.w, ab.z - auxA[i].z);
                        if (lb < best) { best = lb; seed = i; }
                    }
                    if (seed < 0) seed = bc * kCl;
                    seed_lb = best;
                }
                // a seed whose bound cannot lower any of the running minima is not
                // queued (after the first chunk pair the minima are usually tight);
                // the cull below then tests that pair exactly like any other
                bool sq = bval && want_seed;
                if (sq && seed >= 0) {
                    const float4 xs = auxA[seed];
                    const float thr = fmaxf(bd, fmaxf(bl + xs.x + ab.x, bh - xs.y - ab.y));
                    sq = seed_lb < thr;
                }
                if (!sq) seed = -1;
                const unsigned sqm = __ballot_sync(0xffffffffu, sq);
                int qn = __popc(sqm);
                if (sq) queue[__popc(sqm & lt_mask)] = (unsigned short)((seed << 8) | lane);
                bool flush = true;
                // cull into the queue, drain 32 pairs at a time; the one evaluation
                // site below keeps the kernel's code small
                int i = 0;
                bool kc = false;
                for (;;) {
                    while (!flush && qn < 16 && i < ca) {
                        if ((i & (kCl - 1)) == 0) {
                            kc = false;
                            if (bval) {
                                const float4 s = clS[i / kCl], a = clA[i / kCl];
                                const float thr = fmaxf(bd, fmaxf(bl + a.x + ab.x, bh - a.y - ab.y));
                                const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                                const float reach = s.w + sb.w + thr;
                                kc = ab.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach;
                            }
                            if (!__any_sync(0xffffffffu, kc)) {
                                i += kCl;
                                continue;
                            }
                        }
                        bool keep = false;
                        if (kc && i != seed) {
                            const float4 s = sphA[i], a = auxA[i];
                            const float thr = fmaxf(bd, fmaxf(bl + a.x + ab.x, bh - a.y - ab.y));
                            const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                            const float reach = s.w + sb.w + thr;
                            keep = ab.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach;
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, keep);
                        if (keep) queue[qn + __popc(m & lt_mask)] = (unsigned short)((i << 8) | lane);
                        qn += __popc(m);
                        ++i;
                    }
                    if (qn == 0) {
                        if (i >= ca) break;  // culled the whole chunk
                        flush = false;       // nothing queued yet (no seed): cull first
                        continue;
                    }
                    // up to 16 pairs per round, two lanes per pair (one half each)
                    const int take = min(qn, 16);
                    __syncwarp();
                    const int pl = lane & 15, part = lane >> 4;
                    float d2 = FLT_MAX;
                    int qi = 0, qj = 0;
                    if (pl < take) {
                        const unsigned e = queue[pl];
                        qi = e >> 8;
                        qj = e & 0xff;
                        PreTri<float> X, Y;
                        load_pre(part ? sB : sA, part ? kCB : kCA, part ? qj : qi, X);
                        load_pre(part ? sA : sB, part ? kCA : kCB, part ? qi : qj, Y);
                        d2 = tri_dist2_half(X, Y, part);
                    }
                    d2 = fminf(d2, __shfl_xor_sync(0xffffffffu, d2, 16));
                    if (pl < take && part == 0) {
                        const float d = sqrtf(d2);
                        const float4 xa = auxA[qi], xb = auxB[qj];
                        bd = fminf(bd, d);
                        bl = fminf(bl, fmaxf(d - xa.x - xb.x, 0.f));
                        bh = fminf(bh, d + xa.y + xb.y);
                        ++full_evals;
                    }
                    bd = warp_min_nonneg(bd);
                    bl = warp_min_nonneg(bl);
                    bh = warp_min_nonneg(bh);
                    qn -= take;
                    const unsigned short moved = lane < qn ? queue[take + lane] : 0;
                    __syncwarp();
                    if (lane < qn) queue[lane] = moved;
                    __syncwarp();
                    flush = false;
                    if (i >= ca && qn == 0) break;
                    if (i >= ca) flush = true;  // last partial batch
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        if (init_bd && !(bd < b_init)) bd = FLT_MAX;  // nothing below the preset bound
        if (lane == 0) out[it] = make_float4(bd, bl, bh, rmax);
        it = __shfl_sync(0xffffffffu, next, 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) full_evals += __shfl_xor_sync(0xffffffffu, full_evals, o);
    if (lane == 0 && n_full) atomicAdd(n_full, full_evals);
}

// ------------------------------------------------------------------ tuned form, lazy staging
// The same algorithm as refine_tuned_kernel (clusters, seed, cull, two-lane
// drain), but only the bounds are staged: per triangle a bounding sphere and
// (ph, h, axis projection), 32 bytes instead of the 37-float PreTri.  A lane
// that evaluates a queued pair loads the pair's two raw triangle records (L1 /
// L2 hits: the staging just read them) and builds both PreTri in registers,
// relative to the same origin as the staging would have -- so the distances,
// and with them the three minima, are bit-identical.  Shared memory per warp
// drops to about 5 KB, so the A side is staged up to 128 triangles at a time
// and an item needs far fewer chunk pairs (each of which restages B).
template <int CA>
struct LazyLayout {
    static_assert(CA % kCl == 0 && CA <= 256, "A chunk must be whole clusters and fit the queue's 8-bit index");
    static constexpr int kNCl = CA / kCl;
    static constexpr int kOffAuxA = 4 * CA;
    static constexpr int kOffClS = 8 * CA;
    static constexpr int kOffClA = kOffClS + 4 * kNCl;
    static constexpr int kOffAuxB = kOffClA + 4 * kNCl;
    static constexpr int kOffSphB = kOffAuxB + 4 * kCB;    // B spheres (spread cull)
    static constexpr int kOffSeedB = kOffSphB + 4 * kCB;   // each lane's queued seed, -1 for none
    static constexpr int kOffQueue = kOffSeedB + kCB;
    static constexpr int kWarpFloats = kOffQueue + kQueue / 2;
    static_assert(kWarpFloats % 4 == 0 && kOffSphB % 4 == 0, "float4 arrays must stay 16-byte aligned");
    // bulk-copy staging (TMA configurations): the raw 48-byte records of the
    // A chunk and of the B chunk, and the warp's mbarrier
    static constexpr int kOffRawA = kWarpFloats;
    static constexpr int kOffRawB = kOffRawA + 4 * kTriF4 * CA;
    static constexpr int kOffBar = kOffRawB + 4 * kTriF4 * kCB;
    static constexpr int kWarpFloatsTma = kOffBar + 4;
    static_assert(kOffRawA % 4 == 0 && kOffRawB % 4 == 0 && kOffBar % 2 == 0 && kWarpFloatsTma % 4 == 0,
                  "staging must stay 16-byte aligned, the mbarrier 8-byte aligned");
};

// ---- 1-D bulk copies (TMA) into shared memory, completion on an mbarrier ----
// Plain global-to-shared copies of this GPU's own memory: no cluster, no
// multicast.  The size and both addresses are multiples of 16 bytes (whole
// 48-byte triangle records of 16-byte aligned arrays).
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// lane 0: the one arrival of this phase, expecting `bytes`, then the copy
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// wait for phase `parity` of the barrier, at most kMbarTries polls; false on
// giving up (the caller flags it; a copy of valid memory always completes)
constexpr int kMbarTries = 1 << 16;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < kMbarTries; ++i) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Bounds of raw triangle record idx relative to o (the formulas of stage_one /
// tri_sphere): sphere = (centre, radius), aux = (ph, h, projection on u).
__device__ __forceinline__ void lazy_bounds(const float4* __restrict__ tri, size_t idx, float4 o, float3 u,
                                            bool far, float& rmax, float4& sph, float4& aux) {
    const float4* t = tri + idx * kTriF4;
    const float4 t0 = t[0], t1 = t[1], t2 = t[2];
    const V3<float> v[3] = {v3(t0.x - o.x, t0.y - o.y, t0.z - o.z), v3(t1.x - o.x, t1.y - o.y, t1.z - o.z),
                            v3(t2.x - o.x, t2.y - o.y, t2.z - o.z)};
    const float3 c = make_float3((v[0].x + v[1].x + v[2].x) * (1.f / 3.f), (v[0].y + v[1].y + v[2].y) * (1.f / 3.f),
                                 (v[0].z + v[1].z + v[2].z) * (1.f / 3.f));
    float r2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float dx = v[k].x - c.x, dy = v[k].y - c.y, dz = v[k].z - c.z;
        r2 = fmaxf(r2, dx * dx + dy * dy + dz * dz);
        rmax = fmaxf(rmax, fmaxf(fabsf(v[k].x), fmaxf(fabsf(v[k].y), fabsf(v[k].z))));
    }
    const float p0 = v[0].x * u.x + v[0].y * u.y + v[0].z * u.z;
    const float p1 = v[1].x * u.x + v[1].y * u.y + v[1].z * u.z;
    const float p2 = v[2].x * u.x + v[2].y * u.y + v[2].z * u.z;
    const float mg = 1e-5f * (fabsf(p0) + fabsf(p1) + fabsf(p2)) + 1e-6f;
    sph = make_float4(c.x, c.y, c.z, radius_sqrt(r2) * 1.0001f + 1e-6f);
    aux = make_float4(t0.w, t1.w, far ? fminf(p0, fminf(p1, p2)) - mg : fmaxf(p0, fmaxf(p1, p2)) + mg, 0.f);
}

__device__ __forceinline__ void lazy_pre(const float4* __restrict__ t, float4 o, PreTri<float>& P) {
    const float4 t0 = t[0], t1 = t[1], t2 = t[2];
    pretri(P, v3(t0.x - o.x, t0.y - o.y, t0.z - o.z), v3(t1.x - o.x, t1.y - o.y, t1.z - o.z),
           v3(t2.x - o.x, t2.y - o.y, t2.z - o.z));
}

// ONE: a drain round gives each lane a whole queued pair (32 per round) and
// the lane evaluates both halves of it, X = A and X = B, one after the other:
// the same code as the two-lane rounds, so the minima are bit-identical, but
// each pair's two PreTri are built once instead of once per half, and the two
// halves are independent dependency chains the scheduler can interleave.
// SEEDS: only the SEEDS lanes whose seed bound is smallest queue their seed
// (ties by lane); the other lanes' seed pairs go through the cull like any
// other pair, against minima the first seeds have already tightened.  Every
// cull is conservative, so the minima are the same for any SEEDS.
// TMA: each A chunk and each B chunk is first brought into shared memory by
// one 1-D bulk copy (cp.async.bulk, completion on the warp's mbarrier); the
// bounds pass and the evaluations then read the records from shared memory.
// A wait that gives up sets work_counter[1] and leaves the item's results NaN.
// SPREAD: the cull spreads a cluster's member tests over the warp -- one
// test per lane for each (lane that needs the cluster, member) pair, 32 per
// round, reading the B lane's sphere and bounds from shared memory -- instead
// of every lane stepping through the 8 members while most of them need none.
// The same pairs are queued (in another order), so the minima are the same.
// CYL: every cluster and member test also takes the cylinder bound
// (cyl_keep) along the item's axis u, which drops the pairs of two surfaces
// facing each other whose centres are offset sideways; the bound holds for
// every pair of points, so the minima are again the same.
template <int WARPS, int CA, int MINB, bool ONE = false, int SEEDS = 32, bool TMA = false, bool SPREAD = false,
          bool CYL = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) refine_lazy_kernel(const float4* __restrict__ triA,
                                                                    const float4* __restrict__ triB,
                                                                    const RefineItem* __restrict__ items,
                                                                    int n_items_host, const unsigned* n_items_dev,
                                                                    float4* __restrict__ out,
                                                                    unsigned* __restrict__ work_counter,
                                                                    unsigned long long* __restrict__ n_full,
                                                                    const float* __restrict__ init_bd) {
    extern __shared__ __align__(16) float smem[];
    const int n_items = n_items_dev ? (int)*n_items_dev : n_items_host;
    using L = LazyLayout<CA>;
    constexpr int kCA = CA;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* ws = smem + (size_t)wid * (TMA ? L::kWarpFloatsTma : L::kWarpFloats);
    float4* rawA = reinterpret_cast<float4*>(ws + L::kOffRawA);
    float4* rawB = reinterpret_cast<float4*>(ws + L::kOffRawB);
    uint64_t* bar = reinterpret_cast<uint64_t*>(ws + L::kOffBar);
    unsigned phase = 0;
    bool stalled = false;
    if (TMA) {
        if (lane == 0) mbar_init(bar);
        fence_async_shared();
        __syncwarp();
    }
    float4* sphA = reinterpret_cast<float4*>(ws);
    float4* auxA = reinterpret_cast<float4*>(ws + L::kOffAuxA);
    float4* clS = reinterpret_cast<float4*>(ws + L::kOffClS);
    float4* clA = reinterpret_cast<float4*>(ws + L::kOffClA);
    float4* auxB = reinterpret_cast<float4*>(ws + L::kOffAuxB);
    float4* sphB = reinterpret_cast<float4*>(ws + L::kOffSphB);
    int* seedB = reinterpret_cast<int*>(ws + L::kOffSeedB);
    unsigned short* queue = reinterpret_cast<unsigned short*>(ws + L::kOffQueue);
    const unsigned lt_mask = (1u << lane) - 1u;
    unsigned long long full_evals = 0;

    unsigned it = 0;
    if (lane == 0) it = atomicAdd(work_counter, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    while (it < (unsigned)n_items) {
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(work_counter, 1u);
        const RefineItem w = items[it];
        if (w.a_cnt == 0 || w.b_cnt == 0) {
            if (lane == 0) out[it] = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
            it = __shfl_sync(0xffffffffu, next, 0);
            continue;
        }
        const float4 o4 = triA[(size_t)w.a_off * kTriF4];
        float3 u;
        {
            const float4 q = triB[(size_t)w.b_off * kTriF4];
            const float ux = q.x - o4.x, uy = q.y - o4.y, uz = q.z - o4.z;
            const float n2 = ux * ux + uy * uy + uz * uz;
            const float inv = n2 > 0.f ? rsqrtf(n2) : 0.f;
            u = make_float3(ux * inv, uy * inv, uz * inv);
        }
        float bd = FLT_MAX, bl = FLT_MAX, bh = FLT_MAX, rmax = 0.f;
        float b_init = FLT_MAX;
        if (init_bd) {
            b_init = init_bd[it];
            bd = b_init;
            bl = -FLT_MAX;
            bh = -FLT_MAX;
            // item-level reject, as in refine_tuned_kernel: if no pair of
            // (cluster, triangle) bounds is closer than the preset, no
            // triangle pair is, and the item has nothing below it (b_init is
            // the same on every lane, so the branch is uniform)
            const bool need =
                !(b_init < FLT_MAX) || item_may_go_below<CA, CYL>(triA, triB, w, o4, u, bd, sphA, auxA, clS, clA, lane);
            if (!__any_sync(0xffffffffu, need)) {
                if (lane == 0) out[it] = make_float4(FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
                it = __shfl_sync(0xffffffffu, next, 0);
                continue;
            }
        }
        for (uint32_t a0 = 0; a0 < w.a_cnt; a0 += kCA) {
            const int ca = min((uint32_t)kCA, w.a_cnt - a0);
            const int ncl = (ca + kCl - 1) / kCl;
            const float4* tA = triA + ((size_t)w.a_off + a0) * kTriF4;
            __syncwarp();
            if (TMA) {
                // every lane is done with the previous chunk's records
                if (lane == 0) {
                    fence_async_shared();
                    bulk_load(rawA, tA, (unsigned)ca * kTriF4 * 16u, bar);
                }
                const bool ok = mbar_wait(bar, phase);
                phase ^= 1u;
                if (__any_sync(0xffffffffu, !ok)) {
                    stalled = true;
                    break;
                }
                tA = rawA;
            }
            for (int k = lane; k < ca; k += 32) lazy_bounds(tA, k, o4, u, false, rmax, sphA[k], auxA[k]);
            __syncwarp();
            build_clusters<CA>(sphA, auxA, ca, clS, clA, lane);
            for (uint32_t b0 = 0; b0 < w.b_cnt; b0 += kCB) {
                const int cb = min((uint32_t)kCB, w.b_cnt - b0);
                const float4* tB = triB + ((size_t)w.b_off + b0) * kTriF4;
                __syncwarp();
                if (TMA) {
                    if (lane == 0) {
                        fence_async_shared();
                        bulk_load(rawB, tB, (unsigned)cb * kTriF4 * 16u, bar);
                    }
                    const bool ok = mbar_wait(bar, phase);
                    phase ^= 1u;
                    if (__any_sync(0xffffffffu, !ok)) {
                        stalled = true;
                        break;
                    }
                    tB = rawB;
                }
                const bool bval = lane < cb;
                float4 sb = make_float4(0.f, 0.f, 0.f, 0.f), ab = make_float4(0.f, 0.f, 0.f, 0.f);
                if (bval) {
                    lazy_bounds(tB, lane, o4, u, true, rmax, sb, ab);
                    auxB[lane] = ab;
                    if (SPREAD) sphB[lane] = sb;
                }
                __syncwarp();
                int seed = -1;
                float seed_lb = FLT_MAX;
                const bool want_seed = bd == FLT_MAX || init_bd != nullptr;
                if (bval && want_seed) {
                    float best = FLT_MAX;
                    int bc = 0;
                    for (int c = 0; c < ncl; ++c) {
                        const float4 s = clS[c];
                        const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                        const float lb = fmaxf(approx_len(dx * dx + dy * dy + dz * dz) - s.w - sb.w, ab.z - clA[c].z);
                        if (lb < best) { best = lb; bc = c; }
                    }
                    best = FLT_MAX;
                    const int mend = min(ca, (bc + 1) * kCl);
                    for (int i = bc * kCl; i < mend; ++i) {
                        const float4 s = sphA[i];
                        const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                        const float lb = fmaxf(approx_len(dx * dx + dy * dy + dz * dz) - s.w - sb.w, ab.z - auxA[i].z);
                        if (lb < best) { best = lb; seed = i; }
                    }
                    if (seed < 0) seed = bc * kCl;
                    seed_lb = best;
                }
                bool sq = bval && want_seed;
                if (sq && seed >= 0) {
                    const float4 xs = auxA[seed];
                    const float thr = fmaxf(bd, fmaxf(bl + xs.x + ab.x, bh - xs.y - ab.y));
                    sq = seed_lb < thr;
                }
                if (SEEDS < 32) {
                    // this lane's rank among the queued seeds by (bound, lane)
                    const float key = sq ? seed_lb : FLT_MAX;
                    int rank = 0;
#pragma unroll 8
                    for (int o = 0; o < 32; ++o) {
                        const float k2 = __shfl_sync(0xffffffffu, key, o);
                        rank += (k2 < key) || (k2 == key && o < lane);
                    }
                    sq = sq && rank < SEEDS;
                }
                if (!sq) seed = -1;
                const unsigned sqm = __ballot_sync(0xffffffffu, sq);
                int qn = __popc(sqm);
                if (sq) queue[__popc(sqm & lt_mask)] = (unsigned short)((seed << 8) | lane);
                bool flush = true;
                int i = 0;
                bool kc = false;
                // spread cull: the cluster being expanded (cm: the lanes that
                // need it; t0: tests done) -- i then is its first member
                unsigned cm = 0;
                int t0 = 0;
                if (SPREAD) {
                    seedB[lane] = seed;
                    __syncwarp();
                }
                for (;;) {
                    if (SPREAD) {
                        while (!flush && qn < (ONE ? 32 : 16) && (cm || i < ca)) {
                            if (!cm) {
                                bool need = false;
                                if (bval) {
                                    const float4 s = clS[i / kCl], a = clA[i / kCl];
                                    const float thr = fmaxf(bd, fmaxf(bl + a.x + ab.x, bh - a.y - ab.y));
                                    const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                                    const float reach = s.w + sb.w + thr;
                                    need = ab.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach &&
                                           (!CYL || cyl_keep(dx, dy, dz, s.w + sb.w, ab.z - a.z, u, thr));
                                }
                                cm = __ballot_sync(0xffffffffu, need);
                                t0 = 0;
                                if (!cm) {
                                    i += kCl;
                                    continue;
                                }
                            }
                            // one round: test t = t0 + lane is member t % 8 for the
                            // (t / 8)-th lane of cm
                            const int nt = __popc(cm) * kCl;
                            const int t = t0 + lane;
                            bool keep = false;
                            int mi = 0, src = 0;
                            if (t < nt) {
                                src = (int)__fns(cm, 0, t / kCl + 1);
                                mi = i + (t & (kCl - 1));
                                if (mi < ca && mi != seedB[src]) {
                                    const float4 s = sphA[mi], a = auxA[mi], sbq = sphB[src], abq = auxB[src];
                                    const float thr = fmaxf(bd, fmaxf(bl + a.x + abq.x, bh - a.y - abq.y));
                                    const float dx = s.x - sbq.x, dy = s.y - sbq.y, dz = s.z - sbq.z;
                                    const float reach = s.w + sbq.w + thr;
                                    keep = abq.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach &&
                                           (!CYL || cyl_keep(dx, dy, dz, s.w + sbq.w, abq.z - a.z, u, thr));
                                }
                            }
                            const unsigned m = __ballot_sync(0xffffffffu, keep);
                            if (keep) queue[qn + __popc(m & lt_mask)] = (unsigned short)((mi << 8) | src);
                            qn += __popc(m);
                            t0 += 32;
                            if (t0 >= nt) {
                                cm = 0;
                                i += kCl;
                            }
                        }
                    } else
                    while (!flush && qn < (ONE ? 32 : 16) && i < ca) {
                        if ((i & (kCl - 1)) == 0) {
                            kc = false;
                            if (bval) {
                                const float4 s = clS[i / kCl], a = clA[i / kCl];
                                const float thr = fmaxf(bd, fmaxf(bl + a.x + ab.x, bh - a.y - ab.y));
                                const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                                const float reach = s.w + sb.w + thr;
                                kc = ab.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach &&
                                     (!CYL || cyl_keep(dx, dy, dz, s.w + sb.w, ab.z - a.z, u, thr));
                            }
                            if (!__any_sync(0xffffffffu, kc)) {
                                i += kCl;
                                continue;
                            }
                        }
                        bool keep = false;
                        if (kc && i != seed) {
                            const float4 s = sphA[i], a = auxA[i];
                            const float thr = fmaxf(bd, fmaxf(bl + a.x + ab.x, bh - a.y - ab.y));
                            const float dx = s.x - sb.x, dy = s.y - sb.y, dz = s.z - sb.z;
                            const float reach = s.w + sb.w + thr;
                            keep = ab.z - a.z < thr && dx * dx + dy * dy + dz * dz < reach * reach &&
                                   (!CYL || cyl_keep(dx, dy, dz, s.w + sb.w, ab.z - a.z, u, thr));
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, keep);
                        if (keep) queue[qn + __popc(m & lt_mask)] = (unsigned short)((i << 8) | lane);
                        qn += __popc(m);
                        ++i;
                    }
                    if (qn == 0) {
                        if (i >= ca && !cm) break;
                        flush = false;
                        continue;
                    }
                    const int take = min(qn, ONE ? 32 : 16);
                    __syncwarp();
                    const int pl = ONE ? lane : lane & 15, part = ONE ? 0 : lane >> 4;
                    float d2 = FLT_MAX;
                    int qi = 0, qj = 0;
                    if (pl < take) {
                        const unsigned e = queue[pl];
                        qi = e >> 8;
                        qj = e & 0xff;
                        PreTri<float> X, Y;
                        if (ONE) {
                            lazy_pre(tA + (size_t)qi * kTriF4, o4, X);
                            lazy_pre(tB + (size_t)qj * kTriF4, o4, Y);
                            d2 = fminf(tri_dist2_half(X, Y, 0), tri_dist2_half(Y, X, 1));
                        } else {
                            lazy_pre(part ? tB + (size_t)qj * kTriF4 : tA + (size_t)qi * kTriF4, o4, X);
                            lazy_pre(part ? tA + (size_t)qi * kTriF4 : tB + (size_t)qj * kTriF4, o4, Y);
                            d2 = tri_dist2_half(X, Y, part);
                        }
                    }
                    if (!ONE) d2 = fminf(d2, __shfl_xor_sync(0xffffffffu, d2, 16));
                    if (pl < take && part == 0) {
                        const float d = sqrtf(d2);
                        const float4 xa = auxA[qi], xb = auxB[qj];
                        bd = fminf(bd, d);
                        bl = fminf(bl, fmaxf(d - xa.x - xb.x, 0.f));
                        bh = fminf(bh, d + xa.y + xb.y);
                        ++full_evals;
                    }
                    bd = warp_min_nonneg(bd);
                    bl = warp_min_nonneg(bl);
                    bh = warp_min_nonneg(bh);
                    qn -= take;
                    const unsigned short moved = lane < qn ? queue[take + lane] : 0;
                    __syncwarp();
                    if (lane < qn) queue[lane] = moved;
                    __syncwarp();
                    flush = false;
                    if (i >= ca && !cm && qn == 0) break;
                    if (i >= ca && !cm) flush = true;
                }
            }
            if (TMA && stalled) break;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        if (init_bd && !(bd < b_init)) bd = FLT_MAX;
        if (TMA && stalled) {
            // a bulk copy did not complete in time: flag it, mark the item
            // NaN and end this warp (its later items are never claimed)
            if (lane == 0) {
                atomicOr(work_counter + 1, 1u);
                const float nan = __int_as_float(0x7fc00000);
                out[it] = make_float4(nan, nan, nan, rmax);
            }
            return;
        }
        if (lane == 0) out[it] = make_float4(bd, bl, bh, rmax);
        it = __shfl_sync(0xffffffffu, next, 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) full_evals += __shfl_xor_sync(0xffffffffu, full_evals, o);
    if (lane == 0 && n_full) atomicAdd(n_full, full_evals);
}

// ------------------------------------------------------------------ launchers
constexpr int kPlainBlock = 256;
constexpr int kTunedWarps = 4;

cudaError_t launch_refine_plain(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                float4* out, cudaStream_t s) {
    if (n_items <= 0) return cudaSuccess;
    int grid = n_items < (1 << 30) ? n_items : (1 << 30);
    refine_plain_kernel<kPlainBlock><<<grid, kPlainBlock, 0, s>>>(triA, triB, items, n_items, out);
    return cudaGetLastError();
}

// The tuned kernel's configurations: A-side triangles staged per warp and
// CTAs per SM (shared memory per warp shrinks with the A chunk, so a smaller
// chunk admits more resident warps).  All give identical results: every pair
// is translated to the same origin and every cull is conservative.
struct TunedCfgDef {
    int chunk_a, ctas_per_sm;
};
// 0-2: PreTri staged in shared memory (refine_tuned_kernel); 3-7: bounds
// staged, PreTri built per evaluated pair (refine_lazy_kernel); 8-9: the lazy
// kernel with one lane per queued pair (both halves in the lane); 10-11: the
// lazy kernel, two lanes and one lane per pair, queuing 8 seeds first;
// 12-13: the lazy kernel staging its raw records by 1-D bulk copies (TMA);
// 14-15: the lazy kernel with 8 seeds first and the spread cull; 16-17: 14-15
// with the cylinder bound in every cull test
constexpr TunedCfgDef kTunedCfgs[kTunedConfigs] = {{64, 3}, {48, 3}, {32, 4}, {128, 3}, {128, 4}, {64, 4},
                                                    {128, 5}, {128, 6}, {128, 4}, {128, 5}, {128, 5}, {128, 5},
                                                    {128, 4}, {64, 5}, {128, 5}, {128, 4}, {128, 5}, {128, 4}};

TunedConfig tuned_config(int cfg) {
    if (cfg < 0 || cfg >= kTunedConfigs) cfg = 0;
    return TunedConfig{kTunedCfgs[cfg].chunk_a, kTunedCfgs[cfg].ctas_per_sm};
}

template <int CA, int MINB>
static cudaError_t launch_tuned_cfg(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                    float4* out, unsigned* work_counter, unsigned long long* n_full, int num_sms,
                                    cudaStream_t s, const unsigned* n_items_dev, const float* init_bd) {
    static bool attr_set[64] = {};  // per device: the attribute belongs to the device's context
    const size_t smem = (size_t)kTunedWarps * TunedLayout<CA>::kWarpFloats * sizeof(float);
    auto kern = refine_tuned_kernel<kTunedWarps, CA, MINB>;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    cudaError_t e = cudaMemsetAsync(work_counter, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    long want = (long)num_sms * MINB;
    long need = ((long)n_items + kTunedWarps - 1) / kTunedWarps;
    int grid = (int)(want < need ? want : need);
    if (grid < 1) grid = 1;
    kern<<<grid, kTunedWarps * 32, smem, s>>>(triA, triB, items, n_items, n_items_dev, out, work_counter, n_full,
                                              init_bd);
    return cudaGetLastError();
}

template <int CA, int MINB, bool ONE = false, int SEEDS = 32, bool TMA = false, bool SPREAD = false,
          bool CYL = false>
static cudaError_t launch_lazy_cfg(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                   float4* out, unsigned* work_counter, unsigned long long* n_full, int num_sms,
                                   cudaStream_t s, const unsigned* n_items_dev, const float* init_bd) {
    const size_t smem = (size_t)kTunedWarps *
                        (TMA ? LazyLayout<CA>::kWarpFloatsTma : LazyLayout<CA>::kWarpFloats) * sizeof(float);
    auto kern = refine_lazy_kernel<kTunedWarps, CA, MINB, ONE, SEEDS, TMA, SPREAD, CYL>;
    if (smem > 48 * 1024) {
        static bool attr_set[64] = {};  // per device
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !attr_set[dev]) {
            const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) attr_set[dev] = true;
        }
    }
    cudaError_t e = cudaMemsetAsync(work_counter, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    long want = (long)num_sms * MINB;
    long need = ((long)n_items + kTunedWarps - 1) / kTunedWarps;
    int grid = (int)(want < need ? want : need);
    if (grid < 1) grid = 1;
    kern<<<grid, kTunedWarps * 32, smem, s>>>(triA, triB, items, n_items, n_items_dev, out, work_counter, n_full,
                                              init_bd);
    return cudaGetLastError();
}

cudaError_t launch_refine_tuned(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                float4* out, unsigned* work_counter, unsigned long long* n_full, int num_sms,
                                int cfg, cudaStream_t s, const unsigned* n_items_dev, const float* init_bd) {
    if (n_items <= 0) return cudaSuccess;
    switch (cfg) {
        case 1: return launch_tuned_cfg<48, 3>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 2: return launch_tuned_cfg<32, 4>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 3: return launch_lazy_cfg<128, 3>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 4: return launch_lazy_cfg<128, 4>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 6: return launch_lazy_cfg<128, 5>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 7: return launch_lazy_cfg<128, 6>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 5: return launch_lazy_cfg<64, 4>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 8: return launch_lazy_cfg<128, 4, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 9: return launch_lazy_cfg<128, 5, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 10: return launch_lazy_cfg<128, 5, false, 8>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 11: return launch_lazy_cfg<128, 5, true, 8>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 12: return launch_lazy_cfg<128, 4, false, 32, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 13: return launch_lazy_cfg<64, 5, false, 32, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 14: return launch_lazy_cfg<128, 5, false, 8, false, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 15: return launch_lazy_cfg<128, 4, false, 8, false, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 16: return launch_lazy_cfg<128, 5, false, 8, false, true, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        case 17: return launch_lazy_cfg<128, 4, false, 8, false, true, true>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
        default: return launch_tuned_cfg<64, 3>(triA, triB, items, n_items, out, work_counter, n_full, num_sms, s, n_items_dev, init_bd);
    }
}

// ------------------------------------------------------------------ FP64 recheck
// Exact (FP64) minimum triangle distance of a few voxel pairs: the tuned form's
// recheck of object pairs whose FP32 decision fell inside the error band.
constexpr int kF64Block = 128;

__global__ void __launch_bounds__(kF64Block) refine_f64_kernel(const float4* __restrict__ triA,
                                                               const float4* __restrict__ triB,
                                                               const RefineItem* __restrict__ items, int n_items_host,
                                                               const unsigned* n_items_dev, double* __restrict__ out) {
    __shared__ double red[kF64Block / 32];
    const int n_items = n_items_dev ? (int)*n_items_dev : n_items_host;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RefineItem w = items[it];
        double best = 1e300;
        if (w.a_cnt && w.b_cnt) {
            const float4 o4 = triA[(size_t)w.a_off * kTriF4];
            const double ox = o4.x, oy = o4.y, oz = o4.z;
            const uint64_t total = (uint64_t)w.a_cnt * w.b_cnt;
            for (uint64_t p = tid; p < total; p += kF64Block) {
                const uint32_t i = (uint32_t)(p / w.b_cnt), j = (uint32_t)(p - (uint64_t)i * w.b_cnt);
                const float4* a = triA + ((size_t)w.a_off + i) * kTriF4;
                const float4* b = triB + ((size_t)w.b_off + j) * kTriF4;
                PreTri<double> A, B;
                pretri(A, v3<double>(a[0].x - ox, a[0].y - oy, a[0].z - oz), v3<double>(a[1].x - ox, a[1].y - oy, a[1].z - oz),
                       v3<double>(a[2].x - ox, a[2].y - oy, a[2].z - oz));
                pretri(B, v3<double>(b[0].x - ox, b[0].y - oy, b[0].z - oz), v3<double>(b[1].x - ox, b[1].y - oy, b[1].z - oz),
                       v3<double>(b[2].x - ox, b[2].y - oy, b[2].z - oz));
                const double d2 = tri_dist2(A, B);
                best = d2 < best ? d2 : best;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double v = __shfl_xor_sync(0xffffffffu, best, o);
            best = v < best ? v : best;
        }
        __syncthreads();
        if (lane == 0) red[wid] = best;
        __syncthreads();
        if (tid == 0) {
            for (int k = 1; k < kF64Block / 32; ++k) best = red[k] < best ? red[k] : best;
            out[it] = (w.a_cnt && w.b_cnt) ? sqrt(best) : 1e300;
        }
    }
}

cudaError_t launch_refine_f64(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                              double* out, cudaStream_t s, const unsigned* n_items_dev) {
    if (n_items <= 0) return cudaSuccess;
    int grid = n_items < 148 * 16 ? n_items : 148 * 16;
    refine_f64_kernel<<<grid, kF64Block, 0, s>>>(triA, triB, items, n_items, n_items_dev, out);
    return cudaGetLastError();
}

// Pack the reference's flat layout (9 floats per triangle + 2 Hausdorff floats)
// into 48-byte triangle records.
__global__ void pack_triangles_kernel(const float* __restrict__ data, const float* __restrict__ hd, size_t n,
                                      float4* __restrict__ tri) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float* d = data + 9 * i;
        float ph = hd ? hd[2 * i] : 0.f, h = hd ? hd[2 * i + 1] : 0.f;
        tri[3 * i + 0] = make_float4(d[0], d[1], d[2], ph);
        tri[3 * i + 1] = make_float4(d[3], d[4], d[5], h);
        tri[3 * i + 2] = make_float4(d[6], d[7], d[8], 0.f);
    }
}

cudaError_t launch_pack_triangles(const float* data, const float* hd, size_t n, float4* tri, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    pack_triangles_kernel<<<(unsigned)blocks, 256, 0, s>>>(data, hd, n, tri);
    return cudaGetLastError();
}

}  // namespace tdp
