// ptdist.cuh -- FP64 point-to-triangle and point-to-box distances for the bound
// preparation kernels (bounds_kernels.cu, built with -fmad=false so that every
// product and sum is rounded on its own).
//
// Point to triangle: the closest point by Voronoi regions of the triangle
// (Ericson, Real-Time Collision Detection, 2005, sec. 5.1.5); a degenerate
// triangle (no positive area in the interior test) is measured by its edges.
#pragma once
#include <cuda_runtime.h>

namespace tdp {
namespace pd {

struct D3 {
    double x, y, z;
};

__host__ __device__ inline D3 sub(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline D3 mad(D3 a, double s, D3 d) { return D3{a.x + s * d.x, a.y + s * d.y, a.z + s * d.z}; }
__host__ __device__ inline double dist(D3 a, D3 b) {
    const D3 d = sub(a, b);
    return sqrt(dot(d, d));
}
__host__ __device__ inline double dmin(double a, double b) { return b < a ? b : a; }
__host__ __device__ inline double dmax(double a, double b) { return b > a ? b : a; }

__host__ __device__ inline double dist2(D3 a, D3 b) {
    const D3 d = sub(a, b);
    return dot(d, d);
}

// squared distance from p to segment ab
__host__ __device__ inline double seg2(D3 p, D3 a, D3 b) {
    const D3 ab = sub(b, a);
    const double den = dot(ab, ab);
    double t = den > 0 ? dot(sub(p, a), ab) / den : 0.0;
    t = t < 0 ? 0.0 : (t > 1 ? 1.0 : t);
    return dist2(p, mad(a, t, ab));
}

// squared distance from p to triangle abc.  The searches compare squared
// distances and take one square root per result: sqrt is monotone and
// correctly rounded, so the root of a max / min of squares is bit for bit
// the max / min of the roots.
__host__ __device__ inline double tri2(D3 p, D3 a, D3 b, D3 c) {
    const D3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return dist2(p, a);  // vertex region a
    const D3 bp = sub(p, b);
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return dist2(p, b);  // vertex region b
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {  // edge ab
        const double den = d1 - d3;
        return dist2(p, mad(a, den > 0 ? d1 / den : 0.0, ab));
    }
    const D3 cp = sub(p, c);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dist2(p, c);  // vertex region c
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {  // edge ac
        const double den = d2 - d6;
        return dist2(p, mad(a, den > 0 ? d2 / den : 0.0, ac));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {  // edge bc
        const double den = (d4 - d3) + (d5 - d6);
        return dist2(p, mad(b, den > 0 ? (d4 - d3) / den : 0.0, sub(c, b)));
    }
    const double s = va + vb + vc;
    if (!(s > 0)) return dmin(seg2(p, a, b), dmin(seg2(p, b, c), seg2(p, c, a)));
    const double v = vb / s, w = vc / s;  // interior: barycentric (1 - v - w, v, w)
    return dist2(p, D3{a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w});
}

// distance from q to the box [lo, hi] (0 inside; +inf for an empty box lo > hi)
__host__ __device__ inline double box_gap(D3 q, float4 lo, float4 hi) {
    const double gx = dmax(dmax((double)lo.x - q.x, q.x - (double)hi.x), 0.0);
    const double gy = dmax(dmax((double)lo.y - q.y, q.y - (double)hi.y), 0.0);
    const double gz = dmax(dmax((double)lo.z - q.z, q.z - (double)hi.z), 0.0);
    return sqrt(gx * gx + gy * gy + gz * gz);
}

// pruning margin around q: far above the FP64 rounding of the distances
// (a few units in the last place of the coordinates), so that a box skipped
// for being farther than the best distance plus this margin cannot hold a
// triangle whose computed distance is the best or ties it
__host__ __device__ inline double margin(D3 q) {
    const double m = dmax(fabs(q.x), dmax(fabs(q.y), fabs(q.z)));
    return 1e-9 * (1.0 + m);
}

}  // namespace pd
}  // namespace tdp
