// oracle/bounds_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement, in FP64, of the per-triangle Hausdorff bounds that the
// product's bound preparation computes on the GPU (tdp_tile_compute_bounds,
// 3dpipe_b200/csrc/bounds_kernels.cu).  The reference computes these bounds by
// sampling in its CGAL preparation step (src/spatial/himesh_hausdorff.cpp:197-270,
// stored per triangle as (proxy, hausdorff) at src/spatial/himesh_retrieve.cpp:131-151);
// the product replaces that step with a conservative rule, restated here:
//
// For an object with LOD-100 facets S (all voxels, stored order) and LOD-l
// triangles T (l = 20..80):
//   ph: every facet s goes to target(s) = the triangle t of T minimising
//       (dist(bary(s), t)^2, index of t); ph(t) = max over s with target t and
//       over the vertices q of s of dist(q, t)  (0 if no facet targets t).
//   h:  e0 = mean edge length of S (edges (0,1),(1,2),(2,0) summed in stored
//       order); t's depth d is the least d < 3 with L / 2^d <= 1.5 e0 (else 3),
//       L its longest edge; t is cut by d midpoint subdivisions into 4^d pieces
//       and h(t) = max over pieces of min over s of max over the piece's three
//       corners c of dist(c, s)  (0 if S is empty).
//   Both are rounded up to float.  Object level: per LOD the max over T of h
//   (hausdorff) and of ph (proxy); LOD 100 is 0 everywhere.
// dist(p, triangle) is the closest-point-by-Voronoi-regions method (Ericson,
// Real-Time Collision Detection, 2005, sec. 5.1.5) with degenerate triangles
// measured by their edges.
//
// `prune` selects a voxel-box pruned search (exact: a voxel is skipped only if
// its box is farther than the best so far plus a margin far above FP64
// rounding) or brute force over every triangle; both give identical bounds.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "rawdt.hpp"

namespace {

struct V3 {
    double x, y, z;
};

inline V3 vsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 vmad(V3 a, double s, V3 d) { return V3{a.x + s * d.x, a.y + s * d.y, a.z + s * d.z}; }
inline double vdist(V3 a, V3 b) {
    const V3 d = vsub(a, b);
    return std::sqrt(vdot(d, d));
}

inline double vdist2(V3 a, V3 b) {
    const V3 d = vsub(a, b);
    return vdot(d, d);
}

double seg_dist2(V3 p, V3 a, V3 b) {
    const V3 ab = vsub(b, a);
    const double den = vdot(ab, ab);
    double t = den > 0 ? vdot(vsub(p, a), ab) / den : 0.0;
    t = t < 0 ? 0.0 : (t > 1 ? 1.0 : t);
    return vdist2(p, vmad(a, t, ab));
}

// squared distance; the searches root it once per result
double tri_dist2(V3 p, V3 a, V3 b, V3 c) {
    const V3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    const double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return vdist2(p, a);
    const V3 bp = vsub(p, b);
    const double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return vdist2(p, b);
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double den = d1 - d3;
        return vdist2(p, vmad(a, den > 0 ? d1 / den : 0.0, ab));
    }
    const V3 cp = vsub(p, c);
    const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return vdist2(p, c);
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double den = d2 - d6;
        return vdist2(p, vmad(a, den > 0 ? d2 / den : 0.0, ac));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
        const double den = (d4 - d3) + (d5 - d6);
        return vdist2(p, vmad(b, den > 0 ? (d4 - d3) / den : 0.0, vsub(c, b)));
    }
    const double s = va + vb + vc;
    if (!(s > 0)) return std::min(seg_dist2(p, a, b), std::min(seg_dist2(p, b, c), seg_dist2(p, c, a)));
    const double v = vb / s, w = vc / s;
    return vdist2(p, V3{a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w});
}

double tri_dist(V3 p, V3 a, V3 b, V3 c) { return std::sqrt(tri_dist2(p, a, b, c)); }

double box_gap(V3 q, const float* lo, const float* hi) {
    const double gx = std::max(std::max((double)lo[0] - q.x, q.x - (double)hi[0]), 0.0);
    const double gy = std::max(std::max((double)lo[1] - q.y, q.y - (double)hi[1]), 0.0);
    const double gz = std::max(std::max((double)lo[2] - q.z, q.z - (double)hi[2]), 0.0);
    return std::sqrt(gx * gx + gy * gy + gz * gz);
}

inline double margin(V3 q) {
    return 1e-9 * (1.0 + std::max(std::fabs(q.x), std::max(std::fabs(q.y), std::fabs(q.z))));
}

float up(double v) {
    float f = (float)v;
    if ((double)f < v) f = std::nextafter(f, INFINITY);
    return f;
}

// One object's triangles at one LOD: flat vertex list, voxel ranges, voxel boxes.
struct Level {
    std::vector<V3> v;               // 3 per triangle
    std::vector<size_t> off;          // [nvox + 1] first triangle of each voxel
    std::vector<float> box;           // [nvox * 6] lo xyz, hi xyz of the voxel's triangles
    size_t n() const { return v.size() / 3; }
};

Level load_level(const oracle::RObject& o, int li) {
    Level L;
    const size_t nv = o.vox.size();
    L.off.assign(nv + 1, 0);
    L.box.assign(nv * 6, 0.f);
    std::vector<float> t, h;
    for (size_t k = 0; k < nv; ++k) {
        o.tris((int)k, li, t, h);
        const size_t n = t.size() / 9;
        float* b = &L.box[k * 6];
        b[0] = b[1] = b[2] = INFINITY;
        b[3] = b[4] = b[5] = -INFINITY;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) {
                const float* p = &t[9 * i + 3 * c];
                L.v.push_back(V3{p[0], p[1], p[2]});
                for (int d = 0; d < 3; ++d) {
                    b[d] = std::min(b[d], p[d]);
                    b[3 + d] = std::max(b[3 + d], p[d]);
                }
            }
        L.off[k + 1] = L.off[k] + n;
    }
    return L;
}

struct Counter {
    double evals = 0;
};

// nearest triangle of T (lexicographic (squared distance, index)) to q; `home` is visited first
size_t nearest(const Level& T, V3 q, size_t home, bool prune, Counter& C) {
    double bd = INFINITY;
    size_t bi = SIZE_MAX;
    auto visit = [&](size_t k) {
        for (size_t i = T.off[k]; i < T.off[k + 1]; ++i) {
            const double d = tri_dist2(q, T.v[3 * i], T.v[3 * i + 1], T.v[3 * i + 2]);
            C.evals += 1;
            if (d < bd || (d == bd && i < bi)) { bd = d; bi = i; }
        }
    };
    const size_t nv = T.off.size() - 1;
    if (!prune) {
        for (size_t k = 0; k < nv; ++k) visit(k);
        return bi;
    }
    const double eps = margin(q);
    visit(home);
    for (size_t k = 0; k < nv; ++k)
        if (k != home && box_gap(q, &T.box[6 * k], &T.box[6 * k + 3]) <= std::sqrt(bd) + eps) visit(k);
    return bi;
}

// min over facets s of S of max over the corners of dist(corner, s)^2
double piece_min(const Level& S, const V3 q[3], size_t home, bool prune, Counter& C) {
    double best = INFINITY;
    auto visit = [&](size_t k) {
        for (size_t i = S.off[k]; i < S.off[k + 1]; ++i) {
            double acc = 0;
            for (int c = 0; c < 3; ++c) {
                const double d = tri_dist2(q[c], S.v[3 * i], S.v[3 * i + 1], S.v[3 * i + 2]);
                C.evals += 1;
                acc = d > acc ? d : acc;
                if (acc >= best) break;
            }
            best = acc < best ? acc : best;
        }
    };
    const size_t nv = S.off.size() - 1;
    if (!prune) {
        for (size_t k = 0; k < nv; ++k) visit(k);
        return best;
    }
    double eps = 0;
    for (int c = 0; c < 3; ++c) eps = std::max(eps, margin(q[c]));
    if (home < nv) visit(home);
    for (size_t k = 0; k < nv; ++k) {
        if (k == home) continue;
        double lb = 0;
        for (int c = 0; c < 3; ++c) lb = std::max(lb, box_gap(q[c], &S.box[6 * k], &S.box[6 * k + 3]));
        if (lb <= std::sqrt(best) + eps) visit(k);
    }
    return best;
}

// barycentric corner weights of the 4^d pieces of a depth-d midpoint subdivision
void pieces(int d, std::vector<V3>& w) {
    w.clear();
    std::vector<V3> cur = {V3{1, 0, 0}, V3{0, 1, 0}, V3{0, 0, 1}};
    for (int lvl = 0; lvl < d; ++lvl) {
        std::vector<V3> nxt;
        for (size_t p = 0; p < cur.size(); p += 3) {
            const V3 a = cur[p], b = cur[p + 1], c = cur[p + 2];
            const V3 ab{(a.x + b.x) * 0.5, (a.y + b.y) * 0.5, (a.z + b.z) * 0.5};
            const V3 bc{(b.x + c.x) * 0.5, (b.y + c.y) * 0.5, (b.z + c.z) * 0.5};
            const V3 ca{(c.x + a.x) * 0.5, (c.y + a.y) * 0.5, (c.z + a.z) * 0.5};
            const V3 kids[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            nxt.insert(nxt.end(), kids, kids + 12);
        }
        cur.swap(nxt);
    }
    w = cur;
}

inline V3 at(V3 w, V3 a, V3 b, V3 c) {
    return V3{a.x * w.x + b.x * w.y + c.x * w.z, a.y * w.x + b.y * w.y + c.y * w.z, a.z * w.x + b.z * w.y + c.z * w.z};
}

// bounds of one object written into `out` (a copy of the tile bytes)
void object_bounds(const oracle::RObject& o, const uint8_t* base, uint8_t* out, bool prune, Counter& C) {
    const size_t nv = o.vox.size();
    const Level S = load_level(o, 4);
    double esum = 0;
    for (size_t i = 0; i < S.n(); ++i) {
        esum += vdist(S.v[3 * i], S.v[3 * i + 1]);
        esum += vdist(S.v[3 * i + 1], S.v[3 * i + 2]);
        esum += vdist(S.v[3 * i + 2], S.v[3 * i]);
    }
    const double e0 = S.n() ? esum / (3.0 * (double)S.n()) : 0.0;
    // voxel of each LOD-100 facet
    std::vector<size_t> svox(S.n());
    for (size_t k = 0; k < nv; ++k)
        for (size_t i = S.off[k]; i < S.off[k + 1]; ++i) svox[i] = k;
    float obj_h[5] = {0, 0, 0, 0, 0}, obj_ph[5] = {0, 0, 0, 0, 0};
    std::vector<V3> w;
    for (int li = 0; li < 5; ++li) {
        std::vector<float> ph, hh;
        if (li < 4) {
            const Level T = load_level(o, li);
            std::vector<double> phd(T.n(), 0.0);
            for (size_t s = 0; s < S.n() && T.n(); ++s) {
                const V3 a = S.v[3 * s], b = S.v[3 * s + 1], c = S.v[3 * s + 2];
                const V3 q{(a.x + b.x + c.x) * (1.0 / 3.0), (a.y + b.y + c.y) * (1.0 / 3.0), (a.z + b.z + c.z) * (1.0 / 3.0)};
                const size_t t = nearest(T, q, svox[s], prune, C);
                if (t == SIZE_MAX) continue;
                double m = 0;
                for (int k = 0; k < 3; ++k) {
                    const double d = tri_dist2(S.v[3 * s + k], T.v[3 * t], T.v[3 * t + 1], T.v[3 * t + 2]);
                    C.evals += 1;
                    m = d > m ? d : m;
                }
                phd[t] = m > phd[t] ? m : phd[t];
            }
            ph.resize(T.n());
            hh.resize(T.n());
            for (size_t k = 0; k < nv; ++k)
                for (size_t t = T.off[k]; t < T.off[k + 1]; ++t) {
                    const V3 a = T.v[3 * t], b = T.v[3 * t + 1], c = T.v[3 * t + 2];
                    const double L = std::max(vdist(a, b), std::max(vdist(b, c), vdist(c, a)));
                    int d = 0;
                    while (d < 3 && L / (double)(1 << d) > 1.5 * e0) ++d;
                    double h = 0;
                    if (S.n()) {
                        pieces(d, w);
                        for (size_t p = 0; p < w.size(); p += 3) {
                            const V3 q[3] = {at(w[p], a, b, c), at(w[p + 1], a, b, c), at(w[p + 2], a, b, c)};
                            const double m = piece_min(S, q, k, prune, C);
                            h = m > h ? m : h;
                        }
                    }
                    ph[t] = up(std::sqrt(phd[t]));
                    hh[t] = up(std::sqrt(h));
                    obj_ph[li] = std::max(obj_ph[li], ph[t]);
                    obj_h[li] = std::max(obj_h[li], hh[t]);
                }
            // write the (proxy, hausdorff) arrays of every voxel at this LOD
            for (size_t k = 0; k < nv; ++k) {
                const oracle::RVoxel& x = o.vox[k];
                uint8_t* dst = out + (o.data - base) + x.off[li] + 36 * x.cnt[li];
                for (size_t i = 0; i < x.cnt[li]; ++i) {
                    const size_t t = T.off[k] + i;
                    std::memcpy(dst + 8 * i, &ph[t], 4);
                    std::memcpy(dst + 8 * i + 4, &hh[t], 4);
                }
            }
        } else {
            for (size_t k = 0; k < nv; ++k) {
                const oracle::RVoxel& x = o.vox[k];
                std::memset(out + (o.data - base) + x.off[4] + 36 * x.cnt[4], 0, 8 * x.cnt[4]);
            }
        }
    }
    // object level (hausdorff, proxy) per LOD, right after the data block's voxel count
    uint64_t ds;
    std::memcpy(&ds, o.data - 8, 8);
    uint8_t* hp = out + (o.data - base) + ds + 8;
    for (int li = 0; li < 5; ++li) {
        std::memcpy(hp + 8 * li, &obj_h[li], 4);
        std::memcpy(hp + 8 * li + 4, &obj_ph[li], 4);
    }
}

}  // namespace

extern "C" {

// Bounds of every object of a RAW tile: `out` receives a copy of the tile with
// every per-triangle (proxy, hausdorff) pair and the object-level values
// replaced.  Returns 0, or -1 for a malformed tile.  *evals (if not NULL) =
// point-triangle distances evaluated.
int tdo_tile_bounds(const uint8_t* raw, size_t len, uint8_t* out, int prune, int threads, double* evals) {
    std::vector<oracle::RObject> objs;
    try {
        objs = oracle::read_tile(raw, len);
    } catch (...) {
        return -1;
    }
    if (out != raw) std::memcpy(out, raw, len);
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<int>(nt, (int)std::max<size_t>(objs.size(), 1));
    std::atomic<size_t> next{0};
    std::vector<Counter> cs(nt);
    std::vector<std::thread> pool;
    for (int k = 0; k < nt; ++k)
        pool.emplace_back([&, k] {
            for (size_t i; (i = next.fetch_add(1)) < objs.size();) object_bounds(objs[i], raw, out, prune != 0, cs[k]);
        });
    for (auto& th : pool) th.join();
    if (evals) {
        double e = 0;
        for (auto& c : cs) e += c.evals;
        *evals = e;
    }
    return 0;
}

// Largest violation of the bounds of a RAW tile over sampled points (FP64):
// out[0] = max over LOD-l triangles t and points x sampled on t of
//          dist(x, S) - h(t);
// out[1] = max over LOD-100 facets s and points y sampled on s of
//          dist(y, T) - max ph over T (the object-level proxy value),
// both over all objects and LODs 20-80; <= 0 means the sampled points obey
// the bounds.  Points: `samples` per triangle, uniform barycentric, seeded.
int tdo_bounds_violation(const uint8_t* raw, size_t len, int samples, uint64_t seed, double out[2]) {
    std::vector<oracle::RObject> objs;
    try {
        objs = oracle::read_tile(raw, len);
    } catch (...) {
        return -1;
    }
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto rnd = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    out[0] = out[1] = -INFINITY;
    std::vector<float> t, h;
    for (const auto& o : objs) {
        const Level S = load_level(o, 4);
        for (int li = 0; li < 4; ++li) {
            const Level T = load_level(o, li);
            std::vector<float> hv;
            float maxph = 0;
            for (size_t k = 0; k < o.vox.size(); ++k) {
                o.tris((int)k, li, t, h);
                for (size_t i = 0; i < t.size() / 9; ++i) {
                    hv.push_back(h[2 * i + 1]);
                    maxph = std::max(maxph, h[2 * i]);
                }
            }
            auto sample = [&](V3 a, V3 b, V3 c) {
                double u = rnd(), v = rnd();
                if (u + v > 1) { u = 1 - u; v = 1 - v; }
                return V3{a.x + u * (b.x - a.x) + v * (c.x - a.x), a.y + u * (b.y - a.y) + v * (c.y - a.y),
                          a.z + u * (b.z - a.z) + v * (c.z - a.z)};
            };
            for (size_t i = 0; i < T.n() && S.n(); ++i)
                for (int r = 0; r < samples; ++r) {
                    const V3 x = sample(T.v[3 * i], T.v[3 * i + 1], T.v[3 * i + 2]);
                    double d = INFINITY;
                    for (size_t s = 0; s < S.n(); ++s) d = std::min(d, tri_dist(x, S.v[3 * s], S.v[3 * s + 1], S.v[3 * s + 2]));
                    out[0] = std::max(out[0], d - (double)hv[i]);
                }
            for (size_t s = 0; s < S.n() && T.n(); ++s)
                for (int r = 0; r < samples; ++r) {
                    const V3 y = sample(S.v[3 * s], S.v[3 * s + 1], S.v[3 * s + 2]);
                    double d = INFINITY;
                    for (size_t i = 0; i < T.n(); ++i) d = std::min(d, tri_dist(y, T.v[3 * i], T.v[3 * i + 1], T.v[3 * i + 2]));
                    out[1] = std::max(out[1], d - (double)maxph);
                }
        }
    }
    return 0;
}

}  // extern "C"
