// cull.cuh -- bounds of triangles and clusters shared by the tuned refine
// (csrc/refine.cu) and the exact-distance stage (csrc/exact_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <float.h>

#include "common.cuh"
#include "tridist.cuh"

namespace tdp {

constexpr int kCB = 32;     // B-side triangles per chunk (one per lane)
constexpr int kCl = 8;      // A-side triangles per cluster

__device__ __forceinline__ float grp8_min(float v) {
#pragma unroll
    for (int o = 1; o < kCl; o <<= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float grp8_max(float v) {
#pragma unroll
    for (int o = 1; o < kCl; o <<= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Cluster records of a staged A chunk of n triangles: clS[c] = sphere holding
// the members' spheres (centre at the middle of their centres' box),
// clA[c] = (largest ph, smallest h, largest projection).
template <int CA>
__device__ __forceinline__ void build_clusters(const float4* sph, const float4* aux, int n, float4* clS, float4* clA,
                                               int lane) {
    for (int base = 0; base < CA; base += 32) {
        const int k = base + lane;
        const bool v = k < n;
        const float4 c = v ? sph[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 a = v ? aux[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float lx = grp8_min(v ? c.x : FLT_MAX), hx = grp8_max(v ? c.x : -FLT_MAX);
        const float ly = grp8_min(v ? c.y : FLT_MAX), hy = grp8_max(v ? c.y : -FLT_MAX);
        const float lz = grp8_min(v ? c.z : FLT_MAX), hz = grp8_max(v ? c.z : -FLT_MAX);
        const float cx = 0.5f * (lx + hx), cy = 0.5f * (ly + hy), cz = 0.5f * (lz + hz);
        float reach = 0.f;
        if (v) {
            const float dx = c.x - cx, dy = c.y - cy, dz = c.z - cz;
            reach = radius_sqrt(dx * dx + dy * dy + dz * dz) + c.w;
        }
        reach = grp8_max(reach);
        const float phx = grp8_max(v ? a.x : 0.f);
        const float hmn = grp8_min(v ? a.y : FLT_MAX);
        const float pmx = grp8_max(v ? a.z : -FLT_MAX);
        if ((lane & (kCl - 1)) == 0 && v) {
            // inflated like the member spheres so rounding never culls a needed pair
            clS[k / kCl] = make_float4(cx, cy, cz, reach * 1.0001f + 1e-5f * (fabsf(cx) + fabsf(cy) + fabsf(cz)) + 1e-6f);
            clA[k / kCl] = make_float4(phx, hmn, pmx, 0.f);
        }
    }
}

// bounding sphere of a triangle record relative to o, inflated like
// tri_sphere (same centre and radius formula, without the PreTri work)
__device__ __forceinline__ float4 quick_sphere(const float4* __restrict__ t, float4 o) {
    const float4 t0 = t[0], t1 = t[1], t2 = t[2];
    const float x0 = t0.x - o.x, y0 = t0.y - o.y, z0 = t0.z - o.z;
    const float x1 = t1.x - o.x, y1 = t1.y - o.y, z1 = t1.z - o.z;
    const float x2 = t2.x - o.x, y2 = t2.y - o.y, z2 = t2.z - o.z;
    const float cx = (x0 + x1 + x2) * (1.f / 3.f), cy = (y0 + y1 + y2) * (1.f / 3.f), cz = (z0 + z1 + z2) * (1.f / 3.f);
    float r2 = (x0 - cx) * (x0 - cx) + (y0 - cy) * (y0 - cy) + (z0 - cz) * (z0 - cz);
    r2 = fmaxf(r2, (x1 - cx) * (x1 - cx) + (y1 - cy) * (y1 - cy) + (z1 - cz) * (z1 - cz));
    r2 = fmaxf(r2, (x2 - cx) * (x2 - cx) + (y2 - cy) * (y2 - cy) + (z2 - cz) * (z2 - cz));
    return make_float4(cx, cy, cz, radius_sqrt(r2) * 1.0001f + 1e-5f * (fabsf(cx) + fabsf(cy) + fabsf(cz)) + 1e-6f);
}

// the triangle's extreme projection on u relative to o (the smallest for far,
// else the largest), widened as lazy_bounds widens it
__device__ __forceinline__ float quick_proj(const float4* __restrict__ t, float4 o, float3 u, bool far) {
    const float4 t0 = t[0], t1 = t[1], t2 = t[2];
    const float p0 = (t0.x - o.x) * u.x + (t0.y - o.y) * u.y + (t0.z - o.z) * u.z;
    const float p1 = (t1.x - o.x) * u.x + (t1.y - o.y) * u.y + (t1.z - o.z) * u.z;
    const float p2 = (t2.x - o.x) * u.x + (t2.y - o.y) * u.y + (t2.z - o.z) * u.z;
    const float mg = 1e-5f * (fabsf(p0) + fabsf(p1) + fabsf(p2)) + 1e-6f;
    return far ? fminf(p0, fminf(p1, p2)) - mg : fmaxf(p0, fmaxf(p1, p2)) + mg;
}

// The item-level test of an item whose minimum is preset to bd: false when no
// (A cluster, B triangle) pair of bounds -- spheres, and with CYL the
// cylinder bound along u -- comes below bd, so that no triangle pair of the
// item does.  The A triangles' spheres go through sphA / auxA and the
// clusters through clS / clA (a warp's staging, CA triangles at a time).

// The bound of a staged chunk of A as a whole: a sphere around its cluster
// spheres and their largest projection on u (inflated like the cluster
// spheres), so that a B triangle far from the whole chunk costs one test
// instead of one per cluster.
struct ChunkBound {
    float4 s;
    float pz;
};

// Stage A triangles [a0, a0 + ca) of item w: spheres and projections on u
// relative to o4, their clusters, and the chunk's bound.
template <int CA, bool CYL>
__device__ __forceinline__ ChunkBound stage_a_chunk(const float4* __restrict__ triA, const RefineItem& w, uint32_t a0,
                                                    int ca, float4 o4, float3 u, float4* sphA, float4* auxA,
                                                    float4* clS, float4* clA, int lane) {
    const int ncl = (ca + kCl - 1) / kCl;
    __syncwarp();
    for (int k = lane; k < ca; k += 32) {
        const float4* t = triA + ((size_t)w.a_off + a0 + k) * kTriF4;
        sphA[k] = quick_sphere(t, o4);
        auxA[k] = make_float4(0.f, 0.f, CYL ? quick_proj(t, o4, u, false) : 0.f, 0.f);
    }
    __syncwarp();
    build_clusters<CA>(sphA, auxA, ca, clS, clA, lane);
    __syncwarp();
    const bool v = lane < ncl;
    const float4 cs = v ? clS[lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    float lx = v ? cs.x : FLT_MAX, hx = v ? cs.x : -FLT_MAX;
    float ly = v ? cs.y : FLT_MAX, hy = v ? cs.y : -FLT_MAX;
    float lz = v ? cs.z : FLT_MAX, hz = v ? cs.z : -FLT_MAX;
    float vz = v ? clA[lane].z : -FLT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
        ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
        hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
        lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
        hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
        vz = fmaxf(vz, __shfl_xor_sync(0xffffffffu, vz, o));
    }
    const float cx = 0.5f * (lx + hx), cy = 0.5f * (ly + hy), cz = 0.5f * (lz + hz);
    float r = 0.f;
    if (v) {
        const float dx = cs.x - cx, dy = cs.y - cy, dz = cs.z - cz;
        r = radius_sqrt(dx * dx + dy * dy + dz * dz) + cs.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
    return ChunkBound{make_float4(cx, cy, cz, r * 1.0001f + 1e-5f * (fabsf(cx) + fabsf(cy) + fabsf(cz)) + 1e-6f), vz};
}

// True (on every lane) when some B triangle of item w and some cluster of
// the staged A chunk (ncl clusters, bound vb) come below bd: every lane
// tests its B triangle; the warp stops at the first chunk of B where any
// lane needs a cluster.
template <bool CYL>
__device__ __forceinline__ bool b_needs_chunk(const float4* __restrict__ triB, const RefineItem& w, int ncl,
                                              const ChunkBound& vb, float4 o4, float3 u, float bd,
                                              const float4* clS, const float4* clA, int lane) {
    bool need = false;
    for (uint32_t b0 = 0; b0 < w.b_cnt; b0 += kCB) {
        if (b0 + lane < w.b_cnt) {
            const float4* t = triB + ((size_t)w.b_off + b0 + lane) * kTriF4;
            const float4 sb = quick_sphere(t, o4);
            const float pb = CYL ? quick_proj(t, o4, u, true) : 0.f;
            const float vx = vb.s.x - sb.x, vy = vb.s.y - sb.y, vw = vb.s.z - sb.z;
            const float vr = vb.s.w + sb.w + bd;
            const bool near = vx * vx + vy * vy + vw * vw < vr * vr &&
                              (!CYL || cyl_keep(vx, vy, vw, vb.s.w + sb.w, pb - vb.pz, u, bd));
            for (int c = 0; near && c < ncl; ++c) {
                const float4 cs = clS[c];
                const float dx = cs.x - sb.x, dy = cs.y - sb.y, dz = cs.z - sb.z;
                const float reach = cs.w + sb.w + bd;
                if (dx * dx + dy * dy + dz * dz < reach * reach &&
                    (!CYL || cyl_keep(dx, dy, dz, cs.w + sb.w, pb - clA[c].z, u, bd))) {
                    need = true;
                    break;
                }
            }
        }
        if (__any_sync(0xffffffffu, need)) return true;
    }
    return false;
}

template <int CA, bool CYL>
__device__ __forceinline__ bool item_may_go_below(const float4* __restrict__ triA, const float4* __restrict__ triB,
                                                  const RefineItem& w, float4 o4, float3 u, float bd, float4* sphA,
                                                  float4* auxA, float4* clS, float4* clA, int lane) {
    for (uint32_t a0 = 0; a0 < w.a_cnt; a0 += CA) {
        const int ca = min((uint32_t)CA, w.a_cnt - a0);
        const ChunkBound vb = stage_a_chunk<CA, CYL>(triA, w, a0, ca, o4, u, sphA, auxA, clS, clA, lane);
        if (b_needs_chunk<CYL>(triB, w, (ca + kCl - 1) / kCl, vb, o4, u, bd, clS, clA, lane)) return true;
    }
    return false;
}

}  // namespace tdp
