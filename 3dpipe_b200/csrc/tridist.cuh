// tridist.cuh -- triangle/triangle minimum distance on the GPU (sm_100a).
//
// Replaces the reference's device TriDist_kernel / TriDist_seg / TriDist_other /
// SegPoints (src/geometry/computing_gpu.cu:158-610).  The value computed is the
// same mathematical quantity (0 when the triangles intersect), but the
// formulation is this project's own, chosen for SIMT execution:
//
//   d(S,T) = 0                              if an edge of one crosses the other
//          = min( 6 vertex->face feet        (only when the foot is interior)
//                 18 vertex->edge distances  (clamped projections)
//                 9  edge/edge interior solutions )
//
// Every candidate is the distance between two actual points of the triangles,
// so rounding can only move the result by a few ulps of the local coordinate
// scale, never by a missed case.  The one ill-conditioned step, the interior
// solution of two nearly parallel edges (sin^2 < kParallelTol), is evaluated in
// FP64 on the spot.  Triangles are pre-processed once (edges, normal, inverse
// lengths, inward side normals) so each pair costs only dot products.
//
// Work per full evaluation (no culling), counted from the code below:
//   kFlopsPerTriPair = 6*28 (vertex->face) + 18*22 (vertex->edge)
//                    + 9*42 (edge/edge interior) + 6*4 (crossing pre-test) = 966
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tdp {

constexpr double kFlopsPerTriPair = 966.0;
constexpr float kParallelTol = 1e-4f;  // sin^2(angle) below which edge/edge goes to FP64

template <typename R> struct V3 { R x, y, z; };

template <typename R> __host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> __host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> __host__ __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R> __host__ __device__ __forceinline__ R clamp01(R v) { return v < R(0) ? R(0) : (v > R(1) ? R(1) : v); }
template <typename R> __host__ __device__ __forceinline__ R fminf_t(R a, R b) { return b < a ? b : a; }

// 1/x.  In FP32 on the device: the hardware's approximate reciprocal
// (rcp.approx.ftz, within an ulp or so) instead of the correctly rounded
// division sequence, which is several dependent instructions on the
// critical path of every evaluation.  Where it scales a parameter (t, s, u
// of a closest point) the point stays on its segment, and the distance at an
// interior minimum moves only to second order; where it scales a squared
// plane distance it adds about an ulp, inside the error bound the join's
// decisions carry.  FP64 and host code divide.
template <typename R> __host__ __device__ __forceinline__ R recip(R x) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4) {
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
#endif
    return R(1) / x;
}

// A triangle with everything the pair test needs that depends on it alone.
template <typename R> struct PreTri {
    V3<R> v[3];    // vertices (already translated to the pair's local origin)
    V3<R> e[3];    // e[k] = v[k+1] - v[k]
    V3<R> n;       // e[0] x e[1]
    R inn;         // 1/|n|^2, 0 for a degenerate triangle
    R ee[3];       // |e[k]|^2
    R iee[3];      // 1/|e[k]|^2, 0 for a degenerate edge
    V3<R> m[3];    // n x e[k]: points into the triangle across edge k
};

template <typename R>
__host__ __device__ __forceinline__ void pretri(PreTri<R>& t, V3<R> a, V3<R> b, V3<R> c) {
    t.v[0] = a; t.v[1] = b; t.v[2] = c;
    t.e[0] = b - a; t.e[1] = c - b; t.e[2] = a - c;
    t.n = cross(t.e[0], t.e[1]);
    R nn = dot(t.n, t.n);
    t.inn = nn > R(0) ? recip(nn) : R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R ee = dot(t.e[k], t.e[k]);
        t.ee[k] = ee;
        t.iee[k] = ee > R(0) ? recip(ee) : R(0);
        t.m[k] = cross(t.n, t.e[k]);
    }
}

// squared distance from p to segment (a, e), e with precomputed 1/|e|^2
template <typename R>
__host__ __device__ __forceinline__ R pt_seg2(V3<R> p, V3<R> a, V3<R> e, R iee) {
    V3<R> w = p - a;
    R t = clamp01(dot(w, e) * iee);
    V3<R> r = w - e * t;
    return dot(r, r);
}

// is point p inside triangle F's prism (foot of perpendicular interior)?
template <typename R>
__host__ __device__ __forceinline__ bool foot_inside(const PreTri<R>& F, V3<R> p) {
    return dot(p - F.v[0], F.m[0]) >= R(0) && dot(p - F.v[1], F.m[1]) >= R(0) &&
           dot(p - F.v[2], F.m[2]) >= R(0);
}

// does edge k of G (heights hG over F's plane) cross F?
template <typename R>
__host__ __device__ __forceinline__ bool edge_crosses(const PreTri<R>& F, const PreTri<R>& G,
                                                      const R* hG, int k) {
    int k1 = (k + 1) % 3;
    R a = hG[k], b = hG[k1];
    if (!((a > R(0) && b < R(0)) || (a < R(0) && b > R(0)))) return false;
    V3<R> p = G.v[k] + G.e[k] * (a / (a - b));
    return foot_inside(F, p);
}

// Interior solution of two edges in FP64 (only for nearly parallel edges).
__host__ __device__ __forceinline__ double edge_pair_interior_f64(V3<double> a, V3<double> e,
                                                                  V3<double> b, V3<double> f) {
    V3<double> g = a - b;
    double ee = dot(e, e), ff = dot(f, f), ef = dot(e, f), eg = dot(e, g), fg = dot(f, g);
    double den = ee * ff - ef * ef;
    if (!(den > 1e-300)) return 1e300;
    double s = (ef * fg - ff * eg) / den;
    double u = (ee * fg - ef * eg) / den;
    if (!(s > 0.0 && s < 1.0 && u > 0.0 && u < 1.0)) return 1e300;
    V3<double> r = (a + e * s) - (b + f * u);
    return dot(r, r);
}

// Interior solution for edge (a,e) of one triangle and (b,f) of the other,
// squared; +inf-like when the closest points of the lines are not interior.
template <typename R>
__host__ __device__ __forceinline__ R edge_pair_interior2(V3<R> a, V3<R> e, R ee, V3<R> b, V3<R> f,
                                                          R ff) {
    V3<R> g = a - b;
    R ef = dot(e, f), eg = dot(e, g), fg = dot(f, g);
    // den/(ee*ff) = sin^2 of the angle between the edges
    R den = ee * ff - ef * ef;
    if (!(den > R(0))) return R(3.0e38);
    if (den < R(kParallelTol) * ee * ff) {
        // nearly parallel: FP64 on the spot (exact conversion of the inputs)
        double r2 = edge_pair_interior_f64(v3<double>(a.x, a.y, a.z), v3<double>(e.x, e.y, e.z),
                                           v3<double>(b.x, b.y, b.z), v3<double>(f.x, f.y, f.z));
        return r2 < 3.0e38 ? R(r2) : R(3.0e38);
    }
    R id = recip(den);
    R s = (ef * fg - ff * eg) * id;
    R u = (ee * fg - ef * eg) * id;
    if (!(s > R(0) && s < R(1) && u > R(0) && u < R(1))) return R(3.0e38);
    V3<R> r = (g + e * s) - f * u;
    return dot(r, r);
}

// Squared minimum distance between two pre-processed triangles.
template <typename R>
__host__ __device__ __forceinline__ R tri_dist2(const PreTri<R>& A, const PreTri<R>& B) {
    R hA[3], hB[3];  // heights of A's vertices over B's plane, B's over A's plane
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        hA[k] = dot(A.v[k] - B.v[0], B.n);
        hB[k] = dot(B.v[k] - A.v[0], A.n);
    }
    // any edge crossing the other triangle -> intersecting
    bool sepA = (hA[0] > R(0) && hA[1] > R(0) && hA[2] > R(0)) || (hA[0] < R(0) && hA[1] < R(0) && hA[2] < R(0));
    bool sepB = (hB[0] > R(0) && hB[1] > R(0) && hB[2] > R(0)) || (hB[0] < R(0) && hB[1] < R(0) && hB[2] < R(0));
    if (!sepA) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (edge_crosses(B, A, hA, k)) return R(0);
    }
    if (!sepB) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (edge_crosses(A, B, hB, k)) return R(0);
    }
    R best = R(3.0e38);
    // vertex -> face
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (B.inn > R(0) && foot_inside(B, A.v[k])) best = fminf_t(best, hA[k] * hA[k] * B.inn);
        if (A.inn > R(0) && foot_inside(A, B.v[k])) best = fminf_t(best, hB[k] * hB[k] * A.inn);
    }
    // vertex -> edge, edge/edge interior
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            best = fminf_t(best, pt_seg2(A.v[i], B.v[j], B.e[j], B.iee[j]));
            best = fminf_t(best, pt_seg2(B.v[i], A.v[j], A.e[j], A.iee[j]));
            best = fminf_t(best, edge_pair_interior2(A.v[i], A.e[i], A.ee[i], B.v[j], B.e[j], B.ee[j]));
        }
    }
    return best;
}

// One half of tri_dist2, for two lanes that evaluate one pair together: the
// lane with part 0 holds (X, Y) = (A, B), the lane with part 1 holds (B, A).
// Each half covers X's three vertex heights, X's edges crossing Y, X's
// vertices onto Y's face and onto Y's edges, and five (part 0) or four (part
// 1) of the nine edge pairs, always evaluated with A's edge first exactly as
// tri_dist2 does; the operands are picked by selects on the part, so both
// halves run the same instructions (no divergence) and the minimum of the two
// halves is bit-identical to tri_dist2(A, B).
template <typename R>
__host__ __device__ __forceinline__ R tri_dist2_half(const PreTri<R>& X, const PreTri<R>& Y, int part) {
    R hX[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) hX[k] = dot(X.v[k] - Y.v[0], Y.n);
    const bool sepX =
        (hX[0] > R(0) && hX[1] > R(0) && hX[2] > R(0)) || (hX[0] < R(0) && hX[1] < R(0) && hX[2] < R(0));
    if (!sepX) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (edge_crosses(Y, X, hX, k)) return R(0);
    }
    R best = R(3.0e38);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (Y.inn > R(0) && foot_inside(Y, X.v[k])) best = fminf_t(best, hX[k] * hX[k] * Y.inn);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) best = fminf_t(best, pt_seg2(X.v[i], Y.v[j], Y.e[j], Y.iee[j]));
    // edge pairs p = 3 i + j (A's edge i, B's edge j): part 0 takes p = 0..4,
    // part 1 takes p = 5..8 (its fifth slot repeats p = 8)
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int p0 = k, p1 = k + 5 < 9 ? k + 5 : 8;
        const int i0 = p0 / 3, j0 = p0 % 3, i1 = p1 / 3, j1 = p1 % 3;
        // A = X for part 0, A = Y for part 1 (and B the other one)
        const V3<R> a = part ? Y.v[i1] : X.v[i0], e = part ? Y.e[i1] : X.e[i0];
        const R ee = part ? Y.ee[i1] : X.ee[i0];
        const V3<R> b = part ? X.v[j1] : Y.v[j0], f = part ? X.e[j1] : Y.e[j0];
        const R ff = part ? X.ee[j1] : Y.ee[j0];
        best = fminf_t(best, edge_pair_interior2(a, e, ee, b, f, ff));
    }
    return best;
}

#ifdef __CUDACC__
__device__ __forceinline__ float approx_len(float d2) { return d2 * rsqrtf(fmaxf(d2, 1e-30f)); }

// Square root of a bounding radius: the hardware's approximation (within an
// ulp or so); every radius it feeds is then inflated by 1e-4 of itself.
__device__ __forceinline__ float radius_sqrt(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Cylinder bound of two triangles (or clusters) with centres d = cA - cB
// apart, radii summing to rsum, and projections on the item's unit axis u
// at least slab apart (<= 0 when they overlap): every pair of their points
// is at least max(slab, 0) apart along u and |d across u| - rsum across it,
// so the pair is kept only when the two together are below thr.  Where the
// surfaces face each other along u this is far tighter than the sphere gap
// |d| - rsum, which spends both radii in the direction of d.  The radii and
// projections carry the staging's inflation, so FP32 rounding never drops a
// pair that could be the minimum.
__device__ __forceinline__ bool cyl_keep(float dx, float dy, float dz, float rsum, float slab, float3 u,
                                         float thr) {
    const float du = dx * u.x + dy * u.y + dz * u.z;
    const float px = dx - du * u.x, py = dy - du * u.y, pz = dz - du * u.z;
    const float lat = fmaxf(approx_len(px * px + py * py + pz * pz) - rsum, 0.f);
    const float sl = fmaxf(slab, 0.f);
    return sl * sl + lat * lat < thr * thr;
}
#endif

}  // namespace tdp
