// gen.cpp -- seeded nuclei/vessel tile generator (see gen.h for what it restates).
//
// Conservative per-triangle bounds.  For a LOD triangle t of object O with
// original (LOD 100) surface S:
//   proxy-hausdorff ph(t): every original facet s is assigned to one LOD
//     triangle t(s) in the same voxel; ph(t) = max over s assigned to t and over
//     the three vertices q of s of dist(q, t).  dist(., t) is convex, so this is
//     the exact max of dist(x, t) over x in s: every surface point lies within
//     ph of the LOD triangle it is assigned to, which makes d - ph1 - ph2 a valid
//     lower bound (reference semantics: src/geometry/computing_gpu.cu:1115-1116).
//   hausdorff h(t): t is split at its edge midpoints into four sub-triangles;
//     each sub-triangle tau is paired with one original facet s(tau) and
//     h(t) = max over tau and its three corners c of dist(c, s(tau)).  Again by
//     convexity this bounds dist(x, S) for every x in t, so d + h1 + h2 is a
//     valid upper bound (reference: computing_gpu.cu:1117).
// The pairings are chosen once on the prototype; each instance evaluates them
// on its own float vertices in double precision and rounds the results up.
#include "storage/gen.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <queue>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "storage/dt_format.h"
#include "tdp.h"

namespace tdp {
namespace {

// ------------------------------------------------------------------ basics
struct Rng {
    uint64_t s;
    Rng(uint64_t seed, uint64_t stream) {
        s = seed * 0x9E3779B97F4A7C15ull ^ (stream + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull;
        next();
        next();
    }
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uni(double a, double b) { return a + (b - a) * uni(); }
    double normal() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct D3 {
    double x = 0, y = 0, z = 0;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 unit(D3 a) {
    double n = norm(a);
    return n > 0 ? a * (1.0 / n) : D3{1, 0, 0};
}

double pt_seg(D3 p, D3 a, D3 b) {
    D3 e = b - a;
    double ee = dot(e, e);
    double t = ee > 0 ? std::clamp(dot(p - a, e) / ee, 0.0, 1.0) : 0.0;
    return norm(p - (a + e * t));
}

// distance from p to triangle abc (closest-point regions, Ericson 2005, sec. 5.1.5)
double pt_tri(D3 p, D3 a, D3 b, D3 c) {
    D3 ab = b - a, ac = c - a;
    if (dot(cross(ab, ac), cross(ab, ac)) < 1e-24 * std::max(1.0, dot(ab, ab) * dot(ac, ac)))
        return std::min(pt_seg(p, a, b), std::min(pt_seg(p, b, c), pt_seg(p, c, a)));
    D3 ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return norm(ap);
    D3 bp = p - b;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return norm(bp);
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return norm(p - (a + ab * (d1 / (d1 - d3))));
    D3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return norm(cp);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return norm(p - (a + ac * (d2 / (d2 - d6))));
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0)
        return norm(p - (b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)))));
    double den = 1.0 / (va + vb + vc);
    return norm(p - (a + ab * (vb * den) + ac * (vc * den)));
}

float round_up(double v) {
    float f = (float)v;
    if ((double)f < v) f = std::nextafter(f, INFINITY);
    return f;
}

using Tri = std::array<int, 3>;

struct Mesh {
    std::vector<D3> V;
    std::vector<Tri> F;
};

// ------------------------------------------------------------------ prototypes
Mesh icosphere(int subdiv) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    Mesh m;
    D3 v[12] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : v) m.V.push_back(unit(p));
    m.F = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
           {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
           {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < subdiv; ++s) {
        std::unordered_map<uint64_t, int> mid;
        auto midpoint = [&](int a, int b) {
            uint64_t key = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            m.V.push_back(unit((m.V[a] + m.V[b]) * 0.5));
            int id = (int)m.V.size() - 1;
            mid[key] = id;
            return id;
        };
        std::vector<Tri> nf;
        for (auto& f : m.F) {
            int a = midpoint(f[0], f[1]), b = midpoint(f[1], f[2]), c = midpoint(f[2], f[0]);
            nf.push_back({f[0], a, c});
            nf.push_back({f[1], b, a});
            nf.push_back({f[2], c, b});
            nf.push_back({a, b, c});
        }
        m.F.swap(nf);
    }
    return m;
}

// Seven closed capped tubes (trunk, 2 level-1 branches, 4 level-2 branches).
// Canonical geometry: segment k along +z at x = 100k, radius 10, nominal length.
constexpr int kSegs = 7;
constexpr double kSegLen[kSegs] = {300, 180, 180, 120, 120, 120, 120};

struct TubeParam {
    std::vector<int> seg;
    std::vector<double> s, theta;  // axial parameter in [0,1], angle
    std::vector<char> on_axis;     // cap centres
};

Mesh tube_set(int M, int R, TubeParam& tp) {
    Mesh m;
    for (int k = 0; k < kSegs; ++k) {
        int base = (int)m.V.size();
        for (int i = 0; i < R; ++i)
            for (int j = 0; j < M; ++j) {
                double th = 6.283185307179586 * j / M, s = (double)i / (R - 1);
                m.V.push_back({100.0 * k + 10 * std::cos(th), 10 * std::sin(th), s * kSegLen[k]});
                tp.seg.push_back(k); tp.s.push_back(s); tp.theta.push_back(th); tp.on_axis.push_back(0);
            }
        int c0 = (int)m.V.size();
        m.V.push_back({100.0 * k, 0, 0});
        tp.seg.push_back(k); tp.s.push_back(0); tp.theta.push_back(0); tp.on_axis.push_back(1);
        int c1 = (int)m.V.size();
        m.V.push_back({100.0 * k, 0, kSegLen[k]});
        tp.seg.push_back(k); tp.s.push_back(1); tp.theta.push_back(0); tp.on_axis.push_back(1);
        auto at = [&](int i, int j) { return base + i * M + (j % M); };
        for (int i = 0; i + 1 < R; ++i)
            for (int j = 0; j < M; ++j) {
                m.F.push_back({at(i, j), at(i, j + 1), at(i + 1, j + 1)});
                m.F.push_back({at(i, j), at(i + 1, j + 1), at(i + 1, j)});
            }
        for (int j = 0; j < M; ++j) {
            m.F.push_back({c0, at(0, j + 1), at(0, j)});
            m.F.push_back({c1, at(R - 1, j), at(R - 1, j + 1)});
        }
    }
    return m;
}

// ------------------------------------------------------------------ decimation
// Half-edge collapse, shortest edge first, with the link condition and a
// normal-flip guard.  Returns the alive triangles at each target count
// (targets in decreasing order); vertices stay original vertices.
std::vector<std::vector<Tri>> decimate(const Mesh& m, const std::vector<size_t>& targets) {
    const int nv = (int)m.V.size();
    std::vector<Tri> F = m.F;
    std::vector<char> falive(F.size(), 1);
    std::vector<std::vector<int>> vf(nv);
    for (int f = 0; f < (int)F.size(); ++f)
        for (int k = 0; k < 3; ++k) vf[F[f][k]].push_back(f);
    std::vector<char> valive(nv, 1);
    std::vector<uint32_t> ver(nv, 0);
    size_t alive = F.size();
    struct E {
        double len;
        int u, v;
        uint32_t vu, vv;
        bool operator>(const E& o) const {
            if (len != o.len) return len > o.len;
            if (u != o.u) return u > o.u;
            return v > o.v;
        }
    };
    std::priority_queue<E, std::vector<E>, std::greater<E>> pq;
    auto push_edges_of = [&](int v) {
        for (int f : vf[v]) {
            if (!falive[f]) continue;
            for (int k = 0; k < 3; ++k) {
                int w = F[f][k];
                if (w == v) continue;
                int a = std::min(v, w), b = std::max(v, w);
                pq.push({dot(m.V[a] - m.V[b], m.V[a] - m.V[b]), a, b, ver[a], ver[b]});
            }
        }
    };
    for (int v = 0; v < nv; ++v) push_edges_of(v);
    auto neighbors = [&](int v) {
        std::vector<int> r;
        for (int f : vf[v])
            if (falive[f])
                for (int k = 0; k < 3; ++k)
                    if (F[f][k] != v) r.push_back(F[f][k]);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        return r;
    };
    auto fnormal = [&](const Tri& t) { return cross(m.V[t[1]] - m.V[t[0]], m.V[t[2]] - m.V[t[0]]); };
    auto try_collapse = [&](int u, int v) -> bool {  // remove u, keep v
        std::vector<int> shared;  // third vertices of faces with both
        for (int f : vf[u])
            if (falive[f]) {
                bool hv = F[f][0] == v || F[f][1] == v || F[f][2] == v;
                if (hv)
                    for (int k = 0; k < 3; ++k)
                        if (F[f][k] != u && F[f][k] != v) shared.push_back(F[f][k]);
            }
        if (shared.size() != 2) return false;
        std::vector<int> nu = neighbors(u), nvv = neighbors(v), common;
        std::set_intersection(nu.begin(), nu.end(), nvv.begin(), nvv.end(), std::back_inserter(common));
        std::sort(shared.begin(), shared.end());
        if (common != shared) return false;
        for (int w : shared)
            if (neighbors(w).size() <= 3) return false;
        for (int f : vf[u]) {
            if (!falive[f]) continue;
            const Tri& t = F[f];
            if (t[0] == v || t[1] == v || t[2] == v) continue;
            Tri n = t;
            for (int k = 0; k < 3; ++k)
                if (n[k] == u) n[k] = v;
            D3 a = fnormal(t), b = fnormal(n);
            double na = norm(a), nb = norm(b);
            if (nb < 1e-12 * (na + 1e-300) || dot(a, b) < 0.3 * na * nb) return false;
        }
        for (int f : vf[u]) {
            if (!falive[f]) continue;
            Tri& t = F[f];
            if (t[0] == v || t[1] == v || t[2] == v) {
                falive[f] = 0;
                --alive;
                continue;
            }
            for (int k = 0; k < 3; ++k)
                if (t[k] == u) t[k] = v;
            vf[v].push_back(f);
        }
        vf[u].clear();
        valive[u] = 0;
        ++ver[u];
        ++ver[v];
        push_edges_of(v);
        return true;
    };
    std::vector<std::vector<Tri>> out;
    size_t ti = 0;
    auto snapshot = [&]() {
        std::vector<Tri> s;
        for (size_t f = 0; f < F.size(); ++f)
            if (falive[f]) s.push_back(F[f]);
        out.push_back(s);
    };
    while (ti < targets.size()) {
        if (alive <= targets[ti]) {
            snapshot();
            ++ti;
            continue;
        }
        if (pq.empty()) {  // cannot go further: keep the coarsest reachable mesh
            snapshot();
            ++ti;
            continue;
        }
        E e = pq.top();
        pq.pop();
        if (!valive[e.u] || !valive[e.v] || ver[e.u] != e.vu || ver[e.v] != e.vv) continue;
        if (!try_collapse(e.u, e.v)) try_collapse(e.v, e.u);
    }
    return out;
}

// ------------------------------------------------------------------ prototype topology
struct Proto {
    Mesh m;                                   // canonical geometry, LOD 100 faces
    int nvox = 0;
    std::vector<Tri> lodF[kNumLods];          // faces per LOD, grouped by voxel
    std::vector<uint32_t> lod_cnt[kNumLods];  // [nvox]
    std::vector<int> core_vertex;             // [nvox]
    // bound pairings for LOD index l < 4 (indices into lodF[4] for LOD-100 facets)
    std::vector<int> ph_target[kNumLods - 1];      // per LOD-100 facet: nearest LOD-l triangle
    std::vector<uint8_t> sub_depth[kNumLods - 1];  // per LOD-l triangle: subdivision depth
    std::vector<uint32_t> sub_off[kNumLods - 1];   // per LOD-l triangle: first sub-triangle (n+1)
    std::vector<int> sub_face[kNumLods - 1];       // per sub-triangle: paired LOD-100 facet
};

D3 bary(const Mesh& m, const Tri& t) { return (m.V[t[0]] + m.V[t[1]] + m.V[t[2]]) * (1.0 / 3.0); }

// Uniform grid over triangle bounding boxes, for nearest-triangle queries.
struct TriGrid {
    D3 lo;
    double cell = 1;
    int n[3] = {1, 1, 1};
    std::vector<std::vector<int>> cells;
    void build(const std::vector<D3>& V, const std::vector<Tri>& F, double cell_) {
        cell = cell_;
        D3 hi = {-1e300, -1e300, -1e300};
        lo = {1e300, 1e300, 1e300};
        for (auto& t : F)
            for (int k = 0; k < 3; ++k) {
                const D3& p = V[t[k]];
                lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
                hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
            }
        n[0] = std::max(1, (int)std::ceil((hi.x - lo.x) / cell) + 1);
        n[1] = std::max(1, (int)std::ceil((hi.y - lo.y) / cell) + 1);
        n[2] = std::max(1, (int)std::ceil((hi.z - lo.z) / cell) + 1);
        cells.assign((size_t)n[0] * n[1] * n[2], {});
        for (int f = 0; f < (int)F.size(); ++f) {
            D3 a = V[F[f][0]], b = a;
            for (int k = 1; k < 3; ++k) {
                const D3& p = V[F[f][k]];
                a = {std::min(a.x, p.x), std::min(a.y, p.y), std::min(a.z, p.z)};
                b = {std::max(b.x, p.x), std::max(b.y, p.y), std::max(b.z, p.z)};
            }
            visit_cells(a, b, [&](size_t c) { cells[c].push_back(f); });
        }
    }
    int ci(double v, double l, int k) const { return std::clamp((int)std::floor((v - l) / cell), 0, n[k] - 1); }
    template <typename Fn>
    void visit_cells(D3 a, D3 b, Fn fn) const {
        int x0 = ci(a.x, lo.x, 0), x1 = ci(b.x, lo.x, 0), y0 = ci(a.y, lo.y, 1), y1 = ci(b.y, lo.y, 1);
        int z0 = ci(a.z, lo.z, 2), z1 = ci(b.z, lo.z, 2);
        for (int x = x0; x <= x1; ++x)
            for (int y = y0; y <= y1; ++y)
                for (int z = z0; z <= z1; ++z) fn(((size_t)x * n[1] + y) * n[2] + z);
    }
    template <typename Fn>
    void visit(D3 a, D3 b, std::vector<int>& stamp, int& tick, Fn fn) const {
        ++tick;
        visit_cells(a, b, [&](size_t c) {
            for (int f : cells[c])
                if (stamp[f] != tick) { stamp[f] = tick; fn(f); }
        });
    }
};

double median_edge(const Mesh& m, const std::vector<Tri>& F) {
    std::vector<double> e;
    for (auto& t : F)
        for (int k = 0; k < 3; ++k) e.push_back(norm(m.V[t[k]] - m.V[t[(k + 1) % 3]]));
    std::nth_element(e.begin(), e.begin() + e.size() / 2, e.end());
    return e[e.size() / 2];
}

// Corners of the sub-triangles of a midpoint subdivision of depth d, as
// barycentric weights on (a, b, c), in a fixed order.
void sub_triangles(int d, std::vector<std::array<D3, 3>>& out) {
    out.clear();
    std::function<void(D3, D3, D3, int)> rec = [&](D3 p, D3 q, D3 r, int k) {
        if (k == 0) { out.push_back({p, q, r}); return; }
        D3 pq = (p + q) * 0.5, qr = (q + r) * 0.5, rp = (r + p) * 0.5;
        rec(p, pq, rp, k - 1);
        rec(q, qr, pq, k - 1);
        rec(r, rp, qr, k - 1);
        rec(pq, qr, rp, k - 1);
    };
    rec({1, 0, 0}, {0, 1, 0}, {0, 0, 1}, d);
}

inline D3 at_bary(D3 w, D3 a, D3 b, D3 c) { return a * w.x + b * w.y + c * w.z; }

void build_proto(Proto& P, int voxel_size, uint64_t seed) {
    const Mesh& m = P.m;
    const size_t nF = m.F.size();
    std::vector<size_t> targets;
    for (int l = kNumLods - 2; l >= 0; --l) targets.push_back(nF * kLods[l] / 100);
    std::vector<std::vector<Tri>> dec = decimate(m, targets);  // 80,60,40,20
    std::vector<Tri> lods[kNumLods];
    lods[kNumLods - 1] = m.F;
    for (int l = 0; l < kNumLods - 1; ++l) lods[l] = dec[kNumLods - 2 - l];

    // skeleton points: farthest-point seeds + 2 Lloyd iterations over vertices
    int nseed = (int)(nF / (size_t)voxel_size) + 1;
    std::vector<D3> seeds;
    std::vector<double> dmin(m.V.size(), 1e300);
    Rng rng(seed, 0xC0FFEE);
    int cur = (int)(rng.next() % m.V.size());
    for (int s = 0; s < nseed; ++s) {
        seeds.push_back(m.V[cur]);
        int far = 0;
        for (size_t i = 0; i < m.V.size(); ++i) {
            dmin[i] = std::min(dmin[i], norm(m.V[i] - m.V[cur]));
            if (dmin[i] > dmin[far]) far = (int)i;
        }
        cur = far;
    }
    for (int it = 0; it < 2; ++it) {
        std::vector<D3> acc(nseed);
        std::vector<int> cnt(nseed, 0);
        for (auto& p : m.V) {
            int best = 0;
            double bd = 1e300;
            for (int s = 0; s < nseed; ++s) {
                double d = dot(p - seeds[s], p - seeds[s]);
                if (d < bd) { bd = d; best = s; }
            }
            acc[best] = acc[best] + p;
            cnt[best]++;
        }
        for (int s = 0; s < nseed; ++s)
            if (cnt[s]) seeds[s] = acc[s] * (1.0 / cnt[s]);
    }
    // facets by barycentre -> skeleton point; core = vertex 0 of the facet nearest the point
    std::vector<int> best_face(nseed, -1);
    std::vector<double> best_d(nseed, 1e300);
    for (size_t f = 0; f < nF; ++f) {
        D3 b = bary(m, m.F[f]);
        int g = 0;
        double gd = 1e300;
        for (int s = 0; s < nseed; ++s) {
            double d = dot(b - seeds[s], b - seeds[s]);
            if (d < gd) { gd = d; g = s; }
        }
        if (gd < best_d[g]) { best_d[g] = gd; best_face[g] = (int)f; }
    }
    P.core_vertex.clear();
    for (int s = 0; s < nseed; ++s)
        if (best_face[s] >= 0) P.core_vertex.push_back(m.F[best_face[s]][0]);
    P.nvox = (int)P.core_vertex.size();
    // every LOD: triangle -> voxel with the nearest core by its first vertex
    for (int l = 0; l < kNumLods; ++l) {
        std::vector<int> vox_of(lods[l].size());
        for (size_t f = 0; f < lods[l].size(); ++f) {
            D3 p = m.V[lods[l][f][0]];
            int g = 0;
            double gd = 1e300;
            for (int v = 0; v < P.nvox; ++v) {
                double d = dot(p - m.V[P.core_vertex[v]], p - m.V[P.core_vertex[v]]);
                if (d < gd) { gd = d; g = v; }
            }
            vox_of[f] = g;
        }
        P.lodF[l].clear();
        P.lod_cnt[l].assign(P.nvox, 0);
        std::vector<int> order(lods[l].size());
        for (size_t f = 0; f < order.size(); ++f) order[f] = (int)f;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return vox_of[a] < vox_of[b]; });
        for (int f : order) {
            P.lodF[l].push_back(lods[l][f]);
            P.lod_cnt[l][vox_of[f]]++;
        }
    }
    // bound pairings on the canonical geometry
    const std::vector<Tri>& F100 = P.lodF[kNumLods - 1];
    const double e0 = median_edge(m, F100);
    TriGrid g100;
    g100.build(m.V, F100, 2 * e0);
    std::vector<int> stamp100(F100.size(), 0);
    int tick100 = 0;
    std::vector<std::array<D3, 3>> subs;
    for (int l = 0; l < kNumLods - 1; ++l) {
        const auto& LF = P.lodF[l];
        const double el = median_edge(m, LF);
        TriGrid gl;
        gl.build(m.V, LF, 2 * el);
        std::vector<int> stampl(LF.size(), 0);
        int tickl = 0;
        // ph: each LOD-100 facet -> nearest LOD-l triangle (by its barycentre)
        P.ph_target[l].assign(F100.size(), -1);
        for (size_t s = 0; s < F100.size(); ++s) {
            D3 b = bary(m, F100[s]);
            int best = -1;
            double bd = 1e300;
            for (double r = gl.cell; best < 0 || bd > r; r *= 2) {
                gl.visit(b - D3{r, r, r}, b + D3{r, r, r}, stampl, tickl, [&](int t) {
                    const Tri& T = LF[t];
                    double d = pt_tri(b, m.V[T[0]], m.V[T[1]], m.V[T[2]]);
                    if (d < bd) { bd = d; best = t; }
                });
                if (r > 1e7) break;
            }
            P.ph_target[l][s] = best;
        }
        // h: subdivide each LOD triangle until its pieces are about one original
        // edge long; pair every piece with the LOD-100 facet minimising the
        // largest distance of the piece's corners
        P.sub_depth[l].assign(LF.size(), 0);
        P.sub_off[l].assign(LF.size() + 1, 0);
        P.sub_face[l].clear();
        for (size_t t = 0; t < LF.size(); ++t) {
            const Tri& T = LF[t];
            D3 a = m.V[T[0]], b = m.V[T[1]], c = m.V[T[2]];
            double L = std::max(norm(a - b), std::max(norm(b - c), norm(c - a)));
            int d = 0;
            while (d < 3 && L / (1 << d) > 1.5 * e0) ++d;
            P.sub_depth[l][t] = (uint8_t)d;
            sub_triangles(d, subs);
            for (auto& w : subs) {
                D3 q[3] = {at_bary(w[0], a, b, c), at_bary(w[1], a, b, c), at_bary(w[2], a, b, c)};
                D3 qlo = {std::min({q[0].x, q[1].x, q[2].x}), std::min({q[0].y, q[1].y, q[2].y}), std::min({q[0].z, q[1].z, q[2].z})};
                D3 qhi = {std::max({q[0].x, q[1].x, q[2].x}), std::max({q[0].y, q[1].y, q[2].y}), std::max({q[0].z, q[1].z, q[2].z})};
                int best = -1;
                double bd = 1e300;
                for (double r = e0; best < 0 || bd > r; r *= 2) {
                    g100.visit(qlo - D3{r, r, r}, qhi + D3{r, r, r}, stamp100, tick100, [&](int f) {
                        const Tri& S = F100[f];
                        double worst = 0;
                        for (int k = 0; k < 3 && worst < bd; ++k)
                            worst = std::max(worst, pt_tri(q[k], m.V[S[0]], m.V[S[1]], m.V[S[2]]));
                        if (worst < bd) { bd = worst; best = f; }
                    });
                    if (r > 1e7) break;
                }
                P.sub_face[l].push_back(best);
            }
            P.sub_off[l][t + 1] = (uint32_t)P.sub_face[l].size();
        }
    }
}

// ------------------------------------------------------------------ instances
struct NucleusInst {
    D3 c;
    double ax, ay, az;
    double rot[9];
    double coef[9];
};

struct VesselInst {
    D3 start[kSegs], dir[kSegs], e1[kSegs], e2[kSegs];
    double len[kSegs];
    double r;
};

void random_rotation(Rng& g, double R[9]) {
    double q0 = g.normal(), q1 = g.normal(), q2 = g.normal(), q3 = g.normal();
    double n = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    q0 /= n; q1 /= n; q2 /= n; q3 /= n;
    R[0] = 1 - 2 * (q2 * q2 + q3 * q3); R[1] = 2 * (q1 * q2 - q0 * q3); R[2] = 2 * (q1 * q3 + q0 * q2);
    R[3] = 2 * (q1 * q2 + q0 * q3); R[4] = 1 - 2 * (q1 * q1 + q3 * q3); R[5] = 2 * (q2 * q3 - q0 * q1);
    R[6] = 2 * (q1 * q3 - q0 * q2); R[7] = 2 * (q2 * q3 + q0 * q1); R[8] = 1 - 2 * (q1 * q1 + q2 * q2);
}

double noise_basis(const double* cf, D3 u) {
    const double b[9] = {u.x, u.y, u.z, u.x * u.y, u.y * u.z, u.z * u.x, u.x * u.x - u.y * u.y,
                         3 * u.z * u.z - 1, u.x * u.y * u.z * 3};
    double s = 0;
    for (int k = 0; k < 9; ++k) s += cf[k] * b[k];
    return s;
}

D3 nucleus_vertex(const NucleusInst& n, D3 u, double nscale) {
    double r = 1.0 + 0.1 * noise_basis(n.coef, u) * nscale;
    D3 q = {u.x * n.ax * r, u.y * n.ay * r, u.z * n.az * r};
    return {n.c.x + n.rot[0] * q.x + n.rot[1] * q.y + n.rot[2] * q.z,
            n.c.y + n.rot[3] * q.x + n.rot[4] * q.y + n.rot[5] * q.z,
            n.c.z + n.rot[6] * q.x + n.rot[7] * q.y + n.rot[8] * q.z};
}

void frame(D3 d, D3& e1, D3& e2) {
    D3 a = std::fabs(d.x) < 0.9 ? D3{1, 0, 0} : D3{0, 1, 0};
    e1 = unit(cross(d, a));
    e2 = cross(d, e1);
}

D3 random_dir_near(Rng& g, D3 d, double angle_deg) {
    D3 e1, e2;
    frame(d, e1, e2);
    double a = angle_deg * 3.141592653589793 / 180.0 * g.uni(0.6, 1.0);
    double phi = g.uni(0, 6.283185307179586);
    return unit(d * std::cos(a) + (e1 * std::cos(phi) + e2 * std::sin(phi)) * std::sin(a));
}

VesselInst make_vessel(Rng& g, D3 centre) {
    VesselInst v;
    v.r = g.uni(5.0, 15.0);
    D3 d0 = unit({g.normal(), g.normal(), g.normal()});
    v.len[0] = kSegLen[0];
    v.start[0] = centre - d0 * (0.5 * kSegLen[0]);
    v.dir[0] = d0;
    int parent[kSegs] = {-1, 0, 0, 1, 1, 2, 2};
    for (int k = 1; k < kSegs; ++k) {
        int p = parent[k];
        v.len[k] = kSegLen[k];
        v.start[k] = v.start[p] + v.dir[p] * v.len[p];
        v.dir[k] = random_dir_near(g, v.dir[p], 40.0);
    }
    for (int k = 0; k < kSegs; ++k) frame(v.dir[k], v.e1[k], v.e2[k]);
    return v;
}

D3 vessel_vertex(const VesselInst& v, const TubeParam& tp, int i) {
    int k = tp.seg[i];
    D3 p = v.start[k] + v.dir[k] * (tp.s[i] * v.len[k]);
    if (tp.on_axis[i]) return p;
    return p + (v.e1[k] * std::cos(tp.theta[i]) + v.e2[k] * std::sin(tp.theta[i])) * v.r;
}

// the noise amplitude's normaliser of a nucleus: 1 / max |noise| over the
// prototype's vertices (a function of its coefficients alone, computed only
// for the nuclei a call writes, by the writing thread)
double noise_scale(const NucleusInst& n, const Mesh& proto) {
    double mx = 0;
    for (auto& u : proto.V) mx = std::max(mx, std::fabs(noise_basis(n.coef, u)));
    return mx > 0 ? 1.0 / mx : 0.0;
}

double seg_axis_dist(const VesselInst& v, D3 p) {
    double d = 1e300;
    for (int k = 0; k < kSegs; ++k) d = std::min(d, pt_seg(p, v.start[k], v.start[k] + v.dir[k] * v.len[k]));
    return d;
}

// ------------------------------------------------------------------ serialisation
struct Writer {
    uint8_t* p;
    template <typename T>
    void put(const T& v) {
        std::memcpy(p, &v, sizeof(T));
        p += sizeof(T);
    }
    void putf(const float* f, size_t n) {
        std::memcpy(p, f, n * sizeof(float));
        p += n * sizeof(float);
    }
};

size_t object_bytes(const Proto& P) {
    std::vector<uint32_t> counts;
    for (int l = 0; l < kNumLods; ++l)
        for (int v = 0; v < P.nvox; ++v) counts.push_back(P.lod_cnt[l][v]);
    return raw_object_bytes((uint32_t)P.nvox, counts.data());
}

// Write one object given its float vertices.
void write_object(const Proto& P, const std::vector<float>& Vf, uint8_t* dst) {
    auto vtx = [&](int i) { return D3{Vf[3 * i], Vf[3 * i + 1], Vf[3 * i + 2]}; };
    const std::vector<Tri>& F100 = P.lodF[kNumLods - 1];
    // per LOD triangle bounds
    std::vector<float> ph[kNumLods], hh[kNumLods];
    float obj_h[kNumLods] = {0}, obj_ph[kNumLods] = {0};
    for (int l = 0; l < kNumLods; ++l) {
        ph[l].assign(P.lodF[l].size(), 0.f);
        hh[l].assign(P.lodF[l].size(), 0.f);
        if (l == kNumLods - 1) continue;
        std::vector<double> phd(P.lodF[l].size(), 0.0);
        for (size_t s = 0; s < F100.size(); ++s) {
            int t = P.ph_target[l][s];
            if (t < 0) continue;
            const Tri& T = P.lodF[l][t];
            D3 a = vtx(T[0]), b = vtx(T[1]), c = vtx(T[2]);
            for (int k = 0; k < 3; ++k) phd[t] = std::max(phd[t], pt_tri(vtx(F100[s][k]), a, b, c));
        }
        std::vector<std::array<D3, 3>> subs;
        int cur_depth = -1;
        for (size_t t = 0; t < P.lodF[l].size(); ++t) {
            const Tri& T = P.lodF[l][t];
            D3 a = vtx(T[0]), b = vtx(T[1]), c = vtx(T[2]);
            if (P.sub_depth[l][t] != cur_depth) {
                cur_depth = P.sub_depth[l][t];
                sub_triangles(cur_depth, subs);
            }
            double h = 0;
            for (size_t q = 0; q < subs.size(); ++q) {
                int f = P.sub_face[l][P.sub_off[l][t] + q];
                double worst;
                if (f < 0) {  // no pairing: every point of t is within its longest edge of a vertex on S
                    worst = std::max(norm(a - b), std::max(norm(b - c), norm(c - a)));
                } else {
                    const Tri& S = F100[f];
                    D3 sa = vtx(S[0]), sb = vtx(S[1]), sc = vtx(S[2]);
                    worst = 0;
                    for (int k = 0; k < 3; ++k)
                        worst = std::max(worst, pt_tri(at_bary(subs[q][k], a, b, c), sa, sb, sc));
                }
                h = std::max(h, worst);
            }
            hh[l][t] = round_up(h);
            ph[l][t] = round_up(phd[t]);
            obj_h[l] = std::max(obj_h[l], hh[l][t]);
            obj_ph[l] = std::max(obj_ph[l], ph[l][t]);
        }
    }
    // voxel boxes cover every triangle the voxel holds at any LOD
    std::vector<float> box(6 * P.nvox);
    for (int v = 0; v < P.nvox; ++v) {
        box[6 * v] = box[6 * v + 1] = box[6 * v + 2] = INFINITY;
        box[6 * v + 3] = box[6 * v + 4] = box[6 * v + 5] = -INFINITY;
    }
    Writer w{dst};
    uint8_t* size_pos = w.p;
    w.put((size_t)0);
    uint8_t* data0 = w.p;
    std::vector<uint64_t> off(kNumLods * P.nvox);
    for (int l = 0; l < kNumLods; ++l) {
        size_t t0 = 0;
        for (int v = 0; v < P.nvox; ++v) {
            off[l * P.nvox + v] = (uint64_t)(w.p - data0);
            const uint32_t n = P.lod_cnt[l][v];
            for (uint32_t i = 0; i < n; ++i) {
                const Tri& T = P.lodF[l][t0 + i];
                for (int k = 0; k < 3; ++k) {
                    const float* q = &Vf[3 * T[k]];
                    w.putf(q, 3);
                    for (int d = 0; d < 3; ++d) {
                        box[6 * v + d] = std::min(box[6 * v + d], q[d]);
                        box[6 * v + 3 + d] = std::max(box[6 * v + 3 + d], q[d]);
                    }
                }
            }
            for (uint32_t i = 0; i < n; ++i) {
                float hd2[2] = {ph[l][t0 + i], hh[l][t0 + i]};
                w.putf(hd2, 2);
            }
            t0 += n;
        }
    }
    size_t data_size = (size_t)(w.p - data0);
    std::memcpy(size_pos, &data_size, sizeof(size_t));
    w.put((size_t)P.nvox);
    for (int l = 0; l < kNumLods; ++l) {
        w.put(obj_h[l]);
        w.put(obj_ph[l]);
    }
    for (int v = 0; v < P.nvox; ++v) {
        w.putf(&box[6 * v], 6);
        w.putf(&Vf[3 * P.core_vertex[v]], 3);
        for (int l = 0; l < kNumLods; ++l) {
            w.put((size_t)off[l * P.nvox + v]);
            w.put((size_t)P.lod_cnt[l][v]);
        }
    }
    // transform: the vertex nearest the centre of the object's bounding box
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const size_t nv = Vf.size() / 3;
    for (size_t i = 0; i < nv; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], Vf[3 * i + d]);
            hi[d] = std::max(hi[d], Vf[3 * i + d]);
        }
    float cen[3] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2])};
    size_t bi = 0;
    float bd = INFINITY;
    for (size_t i = 0; i < nv; ++i) {
        float dx = Vf[3 * i] - cen[0], dy = Vf[3 * i + 1] - cen[1], dz = Vf[3 * i + 2] - cen[2];
        float d = dx * dx + dy * dy + dz * dz;
        if (d < bd) { bd = d; bi = i; }
    }
    w.putf(&Vf[3 * bi], 3);
}

template <typename Fn>
void parallel_for(long n, int threads, Fn fn) {
    if (threads <= 1 || n < 2) {
        for (long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<long> next{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t)
        ts.emplace_back([&]() {
            for (long i; (i = next.fetch_add(1)) < n;) fn(i);
        });
    for (auto& t : ts) t.join();
}

}  // namespace

namespace {

struct Protos {
    Proto nuc, ves;
    TubeParam tp;
    int key[5];
};

// prototypes (cached per parameter set) and the placed instances of a tile pair
struct Instances {
    std::shared_ptr<const Protos> protos;
    std::vector<VesselInst> ves;
    std::vector<NucleusInst> nuc;
};

int place_instances(const GenParams& p, std::shared_ptr<const Protos>& PR, std::vector<VesselInst>& ves,
                    std::vector<NucleusInst>& nuc, std::string& err);

// The placed instances of a parameter set, computed once and kept (the last
// set) so that the size query, the write and every later range of the same
// tiles reuse them; they are never modified after placement.
int make_instances(const GenParams& p, std::shared_ptr<const Instances>& out, std::string& err) {
    static std::mutex mu;
    static std::shared_ptr<const Instances> last;
    static GenParams last_p;
    std::lock_guard<std::mutex> g(mu);
    auto same = [&](const GenParams& a, const GenParams& b) {
        return a.n_vessels == b.n_vessels && a.nuclei_per_vessel == b.nuclei_per_vessel && a.seed == b.seed &&
               a.voxel_size == b.voxel_size && a.nucleus_subdiv == b.nucleus_subdiv && a.tube_sides == b.tube_sides &&
               a.tube_rings == b.tube_rings && a.grid == b.grid && a.shell_min == b.shell_min &&
               a.shell_max == b.shell_max;
    };
    if (last && same(p, last_p)) {
        out = last;
        return TDP_OK;
    }
    auto inst = std::make_shared<Instances>();
    const int rc = place_instances(p, inst->protos, inst->ves, inst->nuc, err);
    if (rc != TDP_OK) return rc;
    last = inst;
    last_p = p;
    out = inst;
    return TDP_OK;
}

int place_instances(const GenParams& p, std::shared_ptr<const Protos>& PR, std::vector<VesselInst>& ves,
                    std::vector<NucleusInst>& nuc, std::string& err) {
    if (p.n_vessels <= 0 || p.nuclei_per_vessel < 0 || p.voxel_size <= 0 || p.nucleus_subdiv < 0 ||
        p.nucleus_subdiv > 5 || p.tube_sides < 3 || p.tube_rings < 2) {
        err = "bad generator parameters";
        return TDP_ERR_ARG;
    }
    static std::mutex cache_mu;
    static std::shared_ptr<const Protos> cache;
    {
        std::lock_guard<std::mutex> g(cache_mu);
        int key[5] = {p.voxel_size, p.nucleus_subdiv, p.tube_sides, p.tube_rings, (int)(p.seed & 0x7fffffff)};
        if (!cache || std::memcmp(cache->key, key, sizeof key) != 0) {
            auto c = std::make_shared<Protos>();
            std::memcpy(c->key, key, sizeof key);
            c->nuc.m = icosphere(p.nucleus_subdiv);
            build_proto(c->nuc, p.voxel_size, p.seed);
            c->ves.m = tube_set(p.tube_sides, p.tube_rings, c->tp);
            build_proto(c->ves, p.voxel_size, p.seed + 1);
            cache = std::move(c);
        }
        PR = cache;
    }
    const Proto& PN = PR->nuc;
    const long n_nuc = (long)p.n_vessels * p.nuclei_per_vessel;
    // vessels on a grid of cells p.grid apart
    int gx = (int)std::ceil(std::cbrt((double)p.n_vessels) - 1e-9);
    if (gx < 1) gx = 1;
    ves.assign(p.n_vessels, VesselInst{});
    for (int i = 0; i < p.n_vessels; ++i) {
        Rng g(p.seed, 1000000 + i);
        D3 c = {p.grid * (i % gx + 0.5), p.grid * ((i / gx) % gx + 0.5), p.grid * (i / (gx * gx) + 0.5)};
        ves[i] = make_vessel(g, c);
    }
    // each vessel's axis box: seg_axis_dist(v, c) is at least the distance from
    // c to it, so a vessel whose box is farther than the clearance (plus a
    // margin far above rounding) is skipped without changing any outcome
    std::vector<std::array<double, 6>> vbox(p.n_vessels);
    for (int i = 0; i < p.n_vessels; ++i) {
        std::array<double, 6>& b = vbox[i];
        b = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
        for (int k = 0; k < kSegs; ++k)
            for (const D3 q : {ves[i].start[k], ves[i].start[k] + ves[i].dir[k] * ves[i].len[k]}) {
                b[0] = std::min(b[0], q.x); b[1] = std::min(b[1], q.y); b[2] = std::min(b[2], q.z);
                b[3] = std::max(b[3], q.x); b[4] = std::max(b[4], q.y); b[5] = std::max(b[5], q.z);
            }
    }
    auto box_gap2 = [&](int i, D3 c) {
        const std::array<double, 6>& b = vbox[i];
        const double gx = std::max({b[0] - c.x, c.x - b[3], 0.0}), gy = std::max({b[1] - c.y, c.y - b[4], 0.0});
        const double gz = std::max({b[2] - c.z, c.z - b[5], 0.0});
        return gx * gx + gy * gy + gz * gz;
    };
    // nuclei placement: sequential rejection sampling with a hash grid
    const double nuc_reach = 12.0 * 1.1 + 0.01;  // max semi-axis times max radial noise
    // vessel cells: every vessel is listed (in index order) in each cell of
    // edge p.grid that its axis box, widened by its largest clearance, meets;
    // a point outside that widened box never fails the clearance test, so the
    // test visits only the vessels of the point's cell
    const double vcell = std::max(1.0, (double)p.grid);
    double vlo[3] = {1e300, 1e300, 1e300}, vhi[3] = {-1e300, -1e300, -1e300};
    std::vector<double> widen(p.n_vessels);
    for (int i = 0; i < p.n_vessels; ++i) {
        widen[i] = ves[i].r + nuc_reach + std::max((double)p.shell_min, 5.0) + 1e-3;
        for (int d = 0; d < 3; ++d) {
            vlo[d] = std::min(vlo[d], vbox[i][d] - widen[i]);
            vhi[d] = std::max(vhi[d], vbox[i][3 + d] + widen[i]);
        }
    }
    long vdim[3];
    for (int d = 0; d < 3; ++d) vdim[d] = (long)std::floor((vhi[d] - vlo[d]) / vcell) + 1;
    std::vector<std::vector<int>> vcells((size_t)vdim[0] * vdim[1] * vdim[2]);
    for (int i = 0; i < p.n_vessels; ++i) {
        long c0[3], c1[3];
        for (int d = 0; d < 3; ++d) {
            c0[d] = (long)std::floor((vbox[i][d] - widen[i] - vlo[d]) / vcell);
            c1[d] = (long)std::floor((vbox[i][3 + d] + widen[i] - vlo[d]) / vcell);
        }
        for (long x = c0[0]; x <= c1[0]; ++x)
            for (long y = c0[1]; y <= c1[1]; ++y)
                for (long z = c0[2]; z <= c1[2]; ++z) vcells[((size_t)x * vdim[1] + y) * vdim[2] + z].push_back(i);
    }
    const std::vector<int> no_vessels;
    auto vessels_near = [&](D3 c) -> const std::vector<int>& {
        const double q[3] = {c.x, c.y, c.z};
        long k[3];
        for (int d = 0; d < 3; ++d) {
            const double f = std::floor((q[d] - vlo[d]) / vcell);
            if (!(f >= 0.0) || f >= (double)vdim[d]) return no_vessels;
            k[d] = (long)f;
        }
        return vcells[((size_t)k[0] * vdim[1] + k[1]) * vdim[2] + k[2]];
    };
    nuc.assign(n_nuc, NucleusInst{});
    {
        const double cell = 2 * nuc_reach + 2.0;
        std::unordered_map<uint64_t, std::vector<int>> hash;
        auto key = [&](long x, long y, long z) {
            return ((uint64_t)(x & 0x1fffff) << 42) | ((uint64_t)(y & 0x1fffff) << 21) | (uint64_t)(z & 0x1fffff);
        };
        for (int vi = 0; vi < p.n_vessels; ++vi) {
            Rng g(p.seed, 2000000 + vi);
            const VesselInst& V = ves[vi];
            double total = 0;
            for (int k = 0; k < kSegs; ++k) total += V.len[k];
            for (int j = 0; j < p.nuclei_per_vessel; ++j) {
                NucleusInst n;
                bool ok = false;
                for (int attempt = 0; attempt < 10000 && !ok; ++attempt) {
                    double pick = g.uni(0, total);
                    int k = 0;
                    while (k + 1 < kSegs && pick > V.len[k]) { pick -= V.len[k]; ++k; }
                    D3 axis = V.start[k] + V.dir[k] * std::min(pick, V.len[k]);
                    double phi = g.uni(0, 6.283185307179586);
                    D3 radial = V.e1[k] * std::cos(phi) + V.e2[k] * std::sin(phi);
                    double rho = V.r + nuc_reach + g.uni(p.shell_min, p.shell_max);
                    D3 c = axis + radial * rho;
                    // keep clear of every vessel and every other nucleus
                    bool bad = false;
                    const int wlo = std::max(0, vi - gx * gx - gx - 1), whi = std::min(p.n_vessels, vi + gx * gx + gx + 2);
                    for (int wv : vessels_near(c)) {
                        if (wv < wlo || wv >= whi) continue;
                        const double clear = ves[wv].r + nuc_reach + (wv == vi ? p.shell_min : 5.0);
                        if (box_gap2(wv, c) > (clear + 1e-6) * (clear + 1e-6)) continue;
                        if (seg_axis_dist(ves[wv], c) < clear) { bad = true; break; }
                    }
                    if (bad) continue;
                    long cx = (long)std::floor(c.x / cell), cy = (long)std::floor(c.y / cell), cz = (long)std::floor(c.z / cell);
                    for (long a = -1; a <= 1 && !bad; ++a)
                        for (long b = -1; b <= 1 && !bad; ++b)
                            for (long e = -1; e <= 1 && !bad; ++e) {
                                auto it = hash.find(key(cx + a, cy + b, cz + e));
                                if (it == hash.end()) continue;
                                for (int o : it->second)
                                    if (norm(nuc[o].c - c) < 2 * nuc_reach + 1.0) { bad = true; break; }
                            }
                    if (bad) continue;
                    n.c = c;
                    ok = true;
                }
                if (!ok) {
                    err = "could not place nucleus " + std::to_string(j) + " around vessel " + std::to_string(vi);
                    return TDP_ERR_ARG;
                }
                n.ax = g.uni(8, 12); n.ay = g.uni(8, 12); n.az = g.uni(8, 12);
                random_rotation(g, n.rot);
                for (double& cf : n.coef) cf = g.normal();
                long id = (long)vi * p.nuclei_per_vessel + j;
                nuc[id] = n;
                long cx = (long)std::floor(n.c.x / cell), cy = (long)std::floor(n.c.y / cell), cz = (long)std::floor(n.c.z / cell);
                hash[key(cx, cy, cz)].push_back((int)id);
            }
        }
    }
    return TDP_OK;
}

void nuclei_range(const GenParams& p, long& b, long& e) {
    const long n_nuc = (long)p.n_vessels * p.nuclei_per_vessel;
    b = std::max(0L, std::min(p.nuclei_begin, n_nuc));
    e = p.nuclei_end <= 0 ? n_nuc : std::max(b, std::min(p.nuclei_end, n_nuc));
}

}  // namespace

int gen_tiles(const GenParams& p, uint8_t* nuc_buf, size_t nuc_cap, size_t* nuc_len, uint8_t* ves_buf,
              size_t ves_cap, size_t* ves_len, std::string& err) {
    std::shared_ptr<const Instances> inst;
    int rc = make_instances(p, inst, err);
    if (rc != TDP_OK) return rc;
    const Protos* PR = inst->protos.get();
    const std::vector<VesselInst>& ves = inst->ves;
    const std::vector<NucleusInst>& nuc = inst->nuc;
    const Proto& PN = PR->nuc;
    const Proto& PV = PR->ves;
    const size_t nuc_obj = object_bytes(PN), ves_obj = object_bytes(PV);
    long nb0, nb1;
    nuclei_range(p, nb0, nb1);
    const size_t need_n = 1 + nuc_obj * (size_t)(nb1 - nb0), need_v = 1 + ves_obj * (size_t)p.n_vessels;
    if (nuc_len) *nuc_len = need_n;
    if (ves_len) *ves_len = need_v;
    if (!nuc_buf && !ves_buf) return TDP_OK;
    if ((nuc_buf && nuc_cap < need_n) || (ves_buf && ves_cap < need_v)) {
        err = "generator output buffer too small";
        return TDP_ERR_ARG;
    }
    const int threads = p.threads > 0 ? p.threads : std::max(1u, std::thread::hardware_concurrency());
    if (nuc_buf) {
        nuc_buf[0] = kRawType;
        parallel_for(nb1 - nb0, threads, [&](long j) {
            const long i = nb0 + j;
            const double ns = noise_scale(nuc[i], PN.m);
            std::vector<float> Vf(3 * PN.m.V.size());
            for (size_t k = 0; k < PN.m.V.size(); ++k) {
                D3 q = nucleus_vertex(nuc[i], PN.m.V[k], ns);
                Vf[3 * k] = (float)q.x; Vf[3 * k + 1] = (float)q.y; Vf[3 * k + 2] = (float)q.z;
            }
            write_object(PN, Vf, nuc_buf + 1 + nuc_obj * (size_t)j);
        });
    }
    if (ves_buf) {
        ves_buf[0] = kRawType;
        parallel_for(p.n_vessels, threads, [&](long i) {
            std::vector<float> Vf(3 * PV.m.V.size());
            for (size_t k = 0; k < PV.m.V.size(); ++k) {
                D3 q = vessel_vertex(ves[i], PR->tp, (int)k);
                Vf[3 * k] = (float)q.x; Vf[3 * k + 1] = (float)q.y; Vf[3 * k + 2] = (float)q.z;
            }
            write_object(PV, Vf, ves_buf + 1 + ves_obj * (size_t)i);
        });
    }
    return TDP_OK;
}

int gen_meshes(const GenParams& p, int which, float* V, size_t vcap, int64_t* voff, uint32_t* F, size_t fcap,
               int64_t* foff, size_t* n_vert, size_t* n_face, long* n_obj, std::string& err) {
    if (which != 0 && which != 1) {
        err = "which must be 0 (nuclei) or 1 (vessels)";
        return TDP_ERR_ARG;
    }
    std::shared_ptr<const Instances> inst;
    int rc = make_instances(p, inst, err);
    if (rc != TDP_OK) return rc;
    const Protos* PR = inst->protos.get();
    const std::vector<VesselInst>& ves = inst->ves;
    const std::vector<NucleusInst>& nuc = inst->nuc;
    const Proto& P = which == 0 ? PR->nuc : PR->ves;
    long b = 0, e = p.n_vessels;
    if (which == 0) nuclei_range(p, b, e);
    const long n = e - b;
    const size_t nv = P.m.V.size(), nf = P.m.F.size();
    if (n_vert) *n_vert = nv * (size_t)n;
    if (n_face) *n_face = nf * (size_t)n;
    if (n_obj) *n_obj = n;
    if (!V && !F) return TDP_OK;
    if (!V || !F || !voff || !foff || vcap < 3 * nv * (size_t)n || fcap < 3 * nf * (size_t)n) {
        err = "mesh output buffers too small";
        return TDP_ERR_ARG;
    }
    const int threads = p.threads > 0 ? p.threads : std::max(1u, std::thread::hardware_concurrency());
    parallel_for(n, threads, [&](long j) {
        const long i = b + j;
        const double ns = which == 0 ? noise_scale(nuc[i], P.m) : 0.0;
        float* dst = V + 3 * nv * (size_t)j;
        for (size_t k = 0; k < nv; ++k) {
            const D3 q = which == 0 ? nucleus_vertex(nuc[i], P.m.V[k], ns) : vessel_vertex(ves[i], PR->tp, (int)k);
            dst[3 * k] = (float)q.x; dst[3 * k + 1] = (float)q.y; dst[3 * k + 2] = (float)q.z;
        }
        uint32_t* fd = F + 3 * nf * (size_t)j;
        for (size_t f = 0; f < nf; ++f)
            for (int k = 0; k < 3; ++k) fd[3 * f + k] = (uint32_t)P.m.F[f][k];
    });
    for (long j = 0; j <= n; ++j) {
        voff[j] = (int64_t)(nv * (size_t)j);
        foff[j] = (int64_t)(nf * (size_t)j);
    }
    return TDP_OK;
}

}  // namespace tdp
