/*
 * oracle/tridist.c -- TEST INFRASTRUCTURE ONLY.  This file is the checker for the
 * CUDA triangle-distance kernels; nothing in the product links or calls it.
 *
 * FP64 CPU restatement of the triangle-triangle minimum distance that the
 * reference evaluates on its refine path:
 *   TriDist            src/geometry/computing_cpu.cpp:403-439  (device: computing_gpu.cu:566-610)
 *   TriDist_seg        src/geometry/computing_cpu.cpp:184-253  (device: computing_gpu.cu:300-376)
 *   TriDist_other      src/geometry/computing_cpu.cpp:260-387  (device: computing_gpu.cu:383-549)
 *   SegPoints          src/geometry/computing_cpu.cpp:60-177   (device: computing_gpu.cu:158-293)
 *   MeshDist           src/geometry/computing_cpu.cpp:441-481  (device: computing_gpu.cu:1069-1152)
 *
 * The reference code is the closest-feature test published with PQP
 * (E. Larsen, S. Gottschalk, M. Lin, D. Manocha, "Fast proximity queries with
 * swept sphere volumes", UNC TR99-018, 1999).  The functions below restate that
 * published method in double precision; they are written from the method, not
 * copied.  One deliberate difference: the published method clamps the segment
 * parameter t to [0,1] before deriving u; the reference's SegPoints
 * (computing_cpu.cpp:84-95) does not, which can make it return a distance that is
 * larger than the true one.  The oracle keeps the published clamp, so it returns
 * the true distance; tests/test_oracle_pin.py measures how often the reference
 * differs.
 *
 * tdo_tri_dist_features() is an independent second formulation (minimum over all
 * closest-feature candidates, plus an explicit crossing test) used to cross-check
 * tdo_tri_dist() to ~1e-12 relative in double.
 */
#include <math.h>
#include <float.h>
#include <stddef.h>
#include "oracle.h"

typedef struct { double x, y, z; } v3;

static inline v3 mk(const double *p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline v3 scl(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 crs(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

/* Closest points X (on P + s*A) and Y (on Q + u*B), s,u in [0,1], plus the
 * separating direction VEC that the slab test of the method uses.
 * Restates SegPoints (computing_cpu.cpp:60-177) with the published clamp on s. */
static void seg_points(v3 P, v3 A, v3 Q, v3 B, v3 *X, v3 *Y, v3 *VEC)
{
    v3 T = sub(Q, P);
    double aa = dot(A, A), bb = dot(B, B), ab = dot(A, B);
    double at = dot(A, T), bt = dot(B, T);
    double den = aa * bb - ab * ab;
    double s = (den != 0.0) ? (at * bb - bt * ab) / den : 0.0;
    if (!(s >= 0.0)) s = 0.0;      /* also catches NaN */
    else if (s > 1.0) s = 1.0;
    double u = (bb != 0.0) ? (s * ab - bt) / bb : 0.0;

    if (!(u > 0.0)) {                      /* Y pinned at Q */
        *Y = Q;
        s = (aa != 0.0) ? at / aa : 0.0;
        if (s <= 0.0) { *X = P; *VEC = sub(Q, P); }
        else if (s >= 1.0) { *X = add(P, A); *VEC = sub(Q, *X); }
        else { *X = add(P, scl(A, s)); *VEC = crs(A, crs(T, A)); }
    } else if (u >= 1.0) {                 /* Y pinned at Q + B */
        *Y = add(Q, B);
        s = (aa != 0.0) ? (ab + at) / aa : 0.0;
        if (s <= 0.0) { *X = P; *VEC = sub(*Y, P); }
        else if (s >= 1.0) { *X = add(P, A); *VEC = sub(*Y, *X); }
        else { *X = add(P, scl(A, s)); *VEC = crs(A, crs(sub(*Y, P), A)); }
    } else {                               /* Y interior to Q + u*B */
        *Y = add(Q, scl(B, u));
        if (s <= 0.0) { *X = P; *VEC = crs(B, crs(T, B)); }
        else if (s >= 1.0) { *X = add(P, A); *VEC = crs(B, crs(sub(Q, *X), B)); }
        else {
            *X = add(P, scl(A, s));
            *VEC = crs(A, B);
            if (dot(*VEC, T) < 0.0) *VEC = scl(*VEC, -1.0);
        }
    }
}

/* Vertex-face case of the method (TriDist_other, computing_cpu.cpp:260-387):
 * if the normal of triangle F separates F from triangle G, take G's vertex with
 * the smallest projection and, when its foot lies inside F, that is the answer.
 * Returns the distance, or -1 when the case does not apply. */
static double vertex_face(const v3 F[3], const v3 Fe[3], const v3 G[3], int *shown_disjoint)
{
    v3 n = crs(Fe[0], Fe[1]);
    double nl = dot(n, n);
    if (!(nl > 1e-15)) return -1.0;
    double pr[3];
    for (int k = 0; k < 3; ++k) pr[k] = dot(sub(F[0], G[k]), n);
    int pt = -1;
    if (pr[0] > 0 && pr[1] > 0 && pr[2] > 0) {
        pt = (pr[0] < pr[1]) ? 0 : 1;
        if (pr[2] < pr[pt]) pt = 2;
    } else if (pr[0] < 0 && pr[1] < 0 && pr[2] < 0) {
        pt = (pr[0] > pr[1]) ? 0 : 1;
        if (pr[2] > pr[pt]) pt = 2;
    }
    if (pt < 0) return -1.0;
    *shown_disjoint = 1;
    for (int k = 0; k < 3; ++k) {
        v3 side = crs(n, Fe[k]);
        if (!(dot(sub(G[pt], F[k]), side) > 0.0)) return -1.0;
    }
    /* foot of the perpendicular from G[pt] onto F's plane */
    v3 foot = add(G[pt], scl(n, pr[pt] / nl));
    v3 d = sub(foot, G[pt]);
    return sqrt(dot(d, d));
}

double tdo_tri_dist(const double *S9, const double *T9)
{
    v3 S[3] = {mk(S9), mk(S9 + 3), mk(S9 + 6)};
    v3 T[3] = {mk(T9), mk(T9 + 3), mk(T9 + 6)};
    v3 Se[3], Te[3];
    for (int i = 0; i < 3; ++i) {
        Se[i] = sub(S[(i + 1) % 3], S[i]);
        Te[i] = sub(T[(i + 1) % 3], T[i]);
    }
    int shown_disjoint = 0;
    double mindd = DBL_MAX;

    /* nine edge pairs with the slab test (TriDist_seg, computing_cpu.cpp:184-253) */
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            v3 X, Y, VEC;
            seg_points(S[i], Se[i], T[j], Te[j], &X, &Y, &VEC);
            v3 V = sub(Y, X);
            double dd = dot(V, V);
            if (dd <= mindd) {
                mindd = dd;
                double a = dot(sub(S[(i + 2) % 3], X), VEC);
                double b = dot(sub(T[(j + 2) % 3], Y), VEC);
                if (a <= 0.0 && b >= 0.0) return sqrt(dd);
                double p = dot(V, VEC);
                if (a < 0.0) a = 0.0;
                if (b > 0.0) b = 0.0;
                if (p - a + b > 0.0) shown_disjoint = 1;
            }
        }
    }
    double r = vertex_face(S, Se, T, &shown_disjoint);
    if (r >= 0.0) return r;
    r = vertex_face(T, Te, S, &shown_disjoint);
    if (r >= 0.0) return r;
    return shown_disjoint ? sqrt(mindd) : 0.0;
}

/* ---- independent formulation: min over every closest-feature candidate ---- */

static double pt_seg2(v3 p, v3 a, v3 e)
{
    double ee = dot(e, e);
    double t = (ee > 0.0) ? clamp01(dot(sub(p, a), e) / ee) : 0.0;
    v3 d = sub(p, add(a, scl(e, t)));
    return dot(d, d);
}

/* squared distance from p to triangle F when p's foot is interior, else +inf */
static double pt_face2(v3 p, const v3 F[3], const v3 Fe[3])
{
    v3 n = crs(Fe[0], Fe[1]);
    double nl = dot(n, n);
    if (!(nl > 0.0)) return INFINITY;
    for (int k = 0; k < 3; ++k)
        if (dot(sub(p, F[k]), crs(n, Fe[k])) < 0.0) return INFINITY;
    double h = dot(sub(p, F[0]), n);
    return h * h / nl;
}

/* does segment a->b cross the (closed) triangle F?  non-coplanar crossings only */
static int seg_crosses(v3 a, v3 b, const v3 F[3], const v3 Fe[3])
{
    v3 n = crs(Fe[0], Fe[1]);
    double da = dot(sub(a, F[0]), n), db = dot(sub(b, F[0]), n);
    if ((da > 0 && db > 0) || (da < 0 && db < 0) || (da == 0 && db == 0)) return 0;
    v3 p = add(a, scl(sub(b, a), da / (da - db)));
    for (int k = 0; k < 3; ++k)
        if (dot(sub(p, F[k]), crs(n, Fe[k])) < 0.0) return 0;
    return 1;
}

double tdo_tri_dist_features(const double *S9, const double *T9)
{
    v3 S[3] = {mk(S9), mk(S9 + 3), mk(S9 + 6)};
    v3 T[3] = {mk(T9), mk(T9 + 3), mk(T9 + 6)};
    v3 Se[3], Te[3];
    for (int i = 0; i < 3; ++i) {
        Se[i] = sub(S[(i + 1) % 3], S[i]);
        Te[i] = sub(T[(i + 1) % 3], T[i]);
    }
    for (int i = 0; i < 3; ++i) {
        if (seg_crosses(S[i], S[(i + 1) % 3], T, Te)) return 0.0;
        if (seg_crosses(T[i], T[(i + 1) % 3], S, Se)) return 0.0;
    }
    double best = INFINITY;
    for (int i = 0; i < 3; ++i) {
        double f = pt_face2(S[i], T, Te);
        if (f < best) best = f;
        f = pt_face2(T[i], S, Se);
        if (f < best) best = f;
        for (int j = 0; j < 3; ++j) {
            f = pt_seg2(S[i], T[j], Te[j]);
            if (f < best) best = f;
            f = pt_seg2(T[i], S[j], Se[j]);
            if (f < best) best = f;
            /* interior-interior edge pair */
            v3 A = Se[i], B = Te[j], D = sub(T[j], S[i]);
            double aa = dot(A, A), bb = dot(B, B), ab = dot(A, B);
            double ad = dot(A, D), bd = dot(B, D);
            double den = aa * bb - ab * ab;
            if (den > 1e-30 * aa * bb) {
                double s = (ad * bb - bd * ab) / den;
                double u = (ad * ab - bd * aa) / den;
                if (s > 0.0 && s < 1.0 && u > 0.0 && u < 1.0) {
                    v3 w = sub(add(S[i], scl(A, s)), add(T[j], scl(B, u)));
                    double g = dot(w, w);
                    if (g < best) best = g;
                }
            }
        }
    }
    return sqrt(best);
}

/* One voxel pair at one LOD: the three minima MeshDist returns
 * (computing_cpu.cpp:441-481): distance, min of max(d-ph1-ph2,0), min of d+h1+h2.
 * Triangles are 9 floats, Hausdorff pairs are (proxy, hausdorff) floats. */
void tdo_voxel_pair(const float *tri1, const float *hd1, size_t n1,
                    const float *tri2, const float *hd2, size_t n2, double out[3])
{
    double d_min = INFINITY, lo_min = INFINITY, hi_min = INFINITY;
    double a[9], b[9];
    for (size_t i = 0; i < n1; ++i) {
        for (int k = 0; k < 9; ++k) a[k] = tri1[9 * i + k];
        for (size_t j = 0; j < n2; ++j) {
            for (int k = 0; k < 9; ++k) b[k] = tri2[9 * j + k];
            double d = tdo_tri_dist(a, b);
            if (d < d_min) d_min = d;
            if (hd1 && hd2) {
                double lo = d - (double)hd1[2 * i] - (double)hd2[2 * j];
                if (lo < 0.0) lo = 0.0;
                double hi = d + (double)hd1[2 * i + 1] + (double)hd2[2 * j + 1];
                if (lo < lo_min) lo_min = lo;
                if (hi < hi_min) hi_min = hi;
            }
        }
    }
    out[0] = d_min;
    out[1] = lo_min;
    out[2] = hi_min;
}

/* batch helper: n pairs of triangles -> n distances (both formulations) */
void tdo_tri_dist_batch(const double *S, const double *T, size_t n, double *out_pqp, double *out_feat)
{
    for (size_t i = 0; i < n; ++i) {
        if (out_pqp) out_pqp[i] = tdo_tri_dist(S + 9 * i, T + 9 * i);
        if (out_feat) out_feat[i] = tdo_tri_dist_features(S + 9 * i, T + 9 * i);
    }
}
