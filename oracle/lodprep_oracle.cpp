// oracle/lodprep_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the product's GPU LOD preparation (tdp_raw_from_meshes,
// 3dpipe_b200/csrc/prep_kernels.cu): LOD-100 meshes in, a RAW tile out whose
// per-triangle bounds are zero (the bounds are tdo_tile_bounds' rule, applied
// to this output afterwards).  The reference prepares its tiles with CGAL:
// progressive decimation (src/spatial/himesh_comp.cpp:28-190), skeleton voxels
// (src/spatial/himesh_skeleton.cpp:17-168), LOD triangles to voxels
// (src/spatial/himesh_retrieve.cpp:183-200), RAW writing
// (src/storage/tile_IO.cpp:79-172).  CGAL is absent; the rule restated here
// keeps the definitions the join relies on and makes every step deterministic:
//
// Object with vertices P[0..n) (float, evaluated in double) and facets F[0..m):
//  1. LODs 80, 60, 40, 20: target(l) = floor(m * l / 100).  Half-edge collapse,
//     shortest edge first: a priority queue holds (|P_a - P_b|^2, a, b) for
//     a < b with the versions of a and b when pushed, ordered by (length, a, b);
//     every edge of every facet is pushed at the start.  A popped entry whose
//     vertices changed version since is skipped.  Otherwise u = a is removed
//     into v = b, or if that is refused b into a; a collapse of u into v is
//     refused unless (i) exactly two live facets hold both, with third vertices
//     w1 != w2, (ii) the common neighbours of u and v are exactly {w1, w2},
//     (iii) w1 and w2 each have more than 3 neighbours, and (iv) no live facet
//     of u without v turns: with n0 = its normal, n1 = the normal with u
//     replaced by v, |n1| >= 1e-12 (|n0| + 1e-300) and n0.n1 >= 0.3 |n0| |n1|.
//     A collapse kills the two facets holding u and v, writes v for u in the
//     others, bumps the versions of u and v and pushes every edge of v's live
//     facets.  Before each pop, while the live count is <= the next target (or
//     the queue is empty), that LOD is the live facets in index order.
//  2. Voxels: nseed = m / voxel_size + 1 seeds by farthest point from vertex 0
//     (dmin by |.|, ties to the lowest index), then two Lloyd steps over all
//     vertices (nearest seed by squared distance, ties to the lowest seed;
//     sums in vertex order; seed = sum * (1 / count) when count > 0).  Each
//     LOD-100 facet goes to the seed nearest its barycentre ((p0 + p1 + p2) *
//     (1/3)); a seed's core is vertex 0 of its nearest facet (ties to the
//     lowest facet); seeds without facets give no voxel.
//  3. A LOD-100 triangle goes to the voxel whose core is nearest its first
//     vertex (ties to the lowest voxel); voxels that receive none are dropped,
//     and then every LOD's triangles go the same way to the voxels kept (the
//     LOD-100 assignment does not change), keeping LOD order within a voxel.
//     Voxel boxes cover the voxel's triangles at every LOD.
//  4. The transform is the vertex nearest the centre of the vertices' float
//     bounding box (float arithmetic, ties to the lowest index).
// Returns 0, or -1 - object for a bad object (no vertex, no facet, an index out
// of range or a facet repeating a vertex).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

namespace {

constexpr int kL = 5;
constexpr int kPct[kL] = {20, 40, 60, 80, 100};

struct V3 {
    double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

using Face = std::array<uint32_t, 3>;

struct Entry {
    double len;
    uint32_t a, b, va, vb;
};
struct Later {
    bool operator()(const Entry& x, const Entry& y) const {
        if (x.len != y.len) return x.len > y.len;
        if (x.a != y.a) return x.a > y.a;
        return x.b > y.b;
    }
};

// step 1: faces of LODs 20, 40, 60, 80 (index order)
void decimate(const std::vector<V3>& P, std::vector<Face> F, std::vector<Face> out[kL - 1]) {
    const size_t n = P.size(), m = F.size();
    std::vector<char> live(m, 1);
    std::vector<std::vector<uint32_t>> vf(n);
    for (uint32_t f = 0; f < m; ++f)
        for (int k = 0; k < 3; ++k) vf[F[f][k]].push_back(f);
    std::vector<uint32_t> ver(n, 0);
    std::priority_queue<Entry, std::vector<Entry>, Later> pq;
    auto push_of = [&](uint32_t v) {
        for (uint32_t f : vf[v]) {
            if (!live[f]) continue;
            for (int k = 0; k < 3; ++k) {
                const uint32_t w = F[f][k];
                if (w == v) continue;
                const uint32_t a = std::min(v, w), b = std::max(v, w);
                const V3 d = sub(P[a], P[b]);
                pq.push({dot(d, d), a, b, ver[a], ver[b]});
            }
        }
    };
    for (uint32_t v = 0; v < n; ++v) push_of(v);
    auto nbrs = [&](uint32_t v) {
        std::vector<uint32_t> r;
        for (uint32_t f : vf[v])
            if (live[f])
                for (int k = 0; k < 3; ++k)
                    if (F[f][k] != v) r.push_back(F[f][k]);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        return r;
    };
    auto normal = [&](const Face& t) { return cross(sub(P[t[1]], P[t[0]]), sub(P[t[2]], P[t[0]])); };
    size_t alive = m;
    auto collapse = [&](uint32_t u, uint32_t v) -> bool {  // u into v
        std::vector<uint32_t> third;
        for (uint32_t f : vf[u])
            if (live[f] && (F[f][0] == v || F[f][1] == v || F[f][2] == v))
                for (int k = 0; k < 3; ++k)
                    if (F[f][k] != u && F[f][k] != v) third.push_back(F[f][k]);
        if (third.size() != 2 || third[0] == third[1]) return false;
        std::sort(third.begin(), third.end());
        const std::vector<uint32_t> nu = nbrs(u), nv = nbrs(v);
        std::vector<uint32_t> common;
        std::set_intersection(nu.begin(), nu.end(), nv.begin(), nv.end(), std::back_inserter(common));
        if (common != third) return false;
        for (uint32_t w : third)
            if (nbrs(w).size() <= 3) return false;
        for (uint32_t f : vf[u]) {
            if (!live[f]) continue;
            const Face& t = F[f];
            if (t[0] == v || t[1] == v || t[2] == v) continue;
            Face s = t;
            for (int k = 0; k < 3; ++k)
                if (s[k] == u) s[k] = v;
            const V3 n0 = normal(t), n1 = normal(s);
            const double a0 = std::sqrt(dot(n0, n0)), a1 = std::sqrt(dot(n1, n1));
            if (a1 < 1e-12 * (a0 + 1e-300) || dot(n0, n1) < 0.3 * a0 * a1) return false;
        }
        for (uint32_t f : vf[u]) {
            if (!live[f]) continue;
            Face& t = F[f];
            if (t[0] == v || t[1] == v || t[2] == v) {
                live[f] = 0;
                --alive;
                continue;
            }
            for (int k = 0; k < 3; ++k)
                if (t[k] == u) t[k] = v;
            vf[v].push_back(f);
        }
        vf[u].clear();
        ++ver[u];
        ++ver[v];
        push_of(v);
        return true;
    };
    int li = kL - 2;  // LOD 80 first
    while (li >= 0) {
        const size_t target = m * (size_t)kPct[li] / 100;
        if (alive <= target || pq.empty()) {
            out[li].clear();
            for (uint32_t f = 0; f < m; ++f)
                if (live[f]) out[li].push_back(F[f]);
            --li;
            continue;
        }
        const Entry e = pq.top();
        pq.pop();
        if (ver[e.a] != e.va || ver[e.b] != e.vb) continue;
        if (!collapse(e.a, e.b)) collapse(e.b, e.a);
    }
}

struct Writer {
    uint8_t* p;
    template <typename T>
    void put(T v) {
        std::memcpy(p, &v, sizeof v);
        p += sizeof v;
    }
};

// steps 2-4 and the RAW bytes of one object; returns its size (dst may be null)
size_t prepare(const float* Pf, size_t n, const uint32_t* Fi, size_t m, int voxel_size, uint8_t* dst) {
    std::vector<V3> P(n);
    for (size_t i = 0; i < n; ++i) P[i] = {Pf[3 * i], Pf[3 * i + 1], Pf[3 * i + 2]};
    std::vector<Face> lod[kL];
    lod[kL - 1].resize(m);
    for (size_t f = 0; f < m; ++f) lod[kL - 1][f] = {Fi[3 * f], Fi[3 * f + 1], Fi[3 * f + 2]};
    decimate(P, lod[kL - 1], lod);

    // 2. seeds by farthest point, two Lloyd steps
    const size_t nseed = m / (size_t)voxel_size + 1;
    std::vector<V3> seed;
    std::vector<double> dmin(n, INFINITY);
    size_t cur = 0;
    for (size_t s = 0; s < nseed; ++s) {
        seed.push_back(P[cur]);
        size_t far = 0;
        for (size_t i = 0; i < n; ++i) {
            const V3 d = sub(P[i], P[cur]);
            dmin[i] = std::min(dmin[i], std::sqrt(dot(d, d)));
            if (dmin[i] > dmin[far]) far = i;
        }
        cur = far;
    }
    auto nearest = [&](V3 p, const std::vector<V3>& c, double& best) {
        size_t g = 0;
        best = INFINITY;
        for (size_t s = 0; s < c.size(); ++s) {
            const V3 d = sub(p, c[s]);
            const double x = dot(d, d);
            if (x < best) { best = x; g = s; }
        }
        return g;
    };
    for (int it = 0; it < 2; ++it) {
        std::vector<V3> acc(nseed, V3{0, 0, 0});
        std::vector<size_t> cnt(nseed, 0);
        for (size_t i = 0; i < n; ++i) {
            double b;
            const size_t g = nearest(P[i], seed, b);
            acc[g] = add(acc[g], P[i]);
            ++cnt[g];
        }
        for (size_t s = 0; s < nseed; ++s)
            if (cnt[s]) seed[s] = scale(acc[s], 1.0 / (double)cnt[s]);
    }
    std::vector<long> best_face(nseed, -1);
    std::vector<double> best_d(nseed, INFINITY);
    for (size_t f = 0; f < m; ++f) {
        const Face& t = lod[kL - 1][f];
        const V3 b = scale(add(add(P[t[0]], P[t[1]]), P[t[2]]), 1.0 / 3.0);
        double d;
        const size_t g = nearest(b, seed, d);
        if (d < best_d[g]) { best_d[g] = d; best_face[g] = (long)f; }
    }
    std::vector<uint32_t> core0;
    for (size_t s = 0; s < nseed; ++s)
        if (best_face[s] >= 0) core0.push_back(lod[kL - 1][best_face[s]][0]);
    // 3. voxels that receive no LOD-100 triangle are dropped
    std::vector<V3> coreP(core0.size());
    for (size_t v = 0; v < core0.size(); ++v) coreP[v] = P[core0[v]];
    std::vector<size_t> got(core0.size(), 0);
    for (const Face& t : lod[kL - 1]) {
        double d;
        ++got[nearest(P[t[0]], coreP, d)];
    }
    std::vector<uint32_t> core;
    for (size_t v = 0; v < core0.size(); ++v)
        if (got[v]) core.push_back(core0[v]);
    const size_t nv = core.size();
    coreP.resize(nv);
    for (size_t v = 0; v < nv; ++v) coreP[v] = P[core[v]];

    // triangles to the kept voxels, grouped by voxel in LOD order
    std::vector<std::vector<uint32_t>> byvox[kL];
    size_t data = 0;
    for (int l = 0; l < kL; ++l) {
        byvox[l].assign(nv, {});
        for (uint32_t f = 0; f < lod[l].size(); ++f) {
            double d;
            byvox[l][nearest(P[lod[l][f][0]], coreP, d)].push_back(f);
        }
        data += 44 * lod[l].size();
    }
    const size_t bytes = 8 + data + 8 + 40 + 116 * nv + 12;
    if (!dst) return bytes;

    Writer w{dst};
    w.put((uint64_t)data);
    std::vector<float> box(6 * nv);
    for (size_t v = 0; v < nv; ++v)
        for (int k = 0; k < 3; ++k) {
            box[6 * v + k] = INFINITY;
            box[6 * v + 3 + k] = -INFINITY;
        }
    std::vector<uint64_t> off(kL * nv);
    const uint8_t* d0 = w.p;
    for (int l = 0; l < kL; ++l)
        for (size_t v = 0; v < nv; ++v) {
            off[l * nv + v] = (uint64_t)(w.p - d0);
            for (uint32_t f : byvox[l][v])
                for (int k = 0; k < 3; ++k) {
                    const float* q = Pf + 3 * (size_t)lod[l][f][k];
                    for (int c = 0; c < 3; ++c) {
                        w.put(q[c]);
                        box[6 * v + c] = std::min(box[6 * v + c], q[c]);
                        box[6 * v + 3 + c] = std::max(box[6 * v + 3 + c], q[c]);
                    }
                }
            for (size_t i = 0; i < 2 * byvox[l][v].size(); ++i) w.put(0.f);
        }
    w.put((uint64_t)nv);
    for (int i = 0; i < 2 * kL; ++i) w.put(0.f);
    for (size_t v = 0; v < nv; ++v) {
        for (int k = 0; k < 6; ++k) w.put(box[6 * v + k]);
        for (int k = 0; k < 3; ++k) w.put(Pf[3 * (size_t)core[v] + k]);
        for (int l = 0; l < kL; ++l) {
            w.put(off[l * nv + v]);
            w.put((uint64_t)byvox[l][v].size());
        }
    }
    // 4. transform
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], Pf[3 * i + k]);
            hi[k] = std::max(hi[k], Pf[3 * i + k]);
        }
    const float cx = 0.5f * (lo[0] + hi[0]), cy = 0.5f * (lo[1] + hi[1]), cz = 0.5f * (lo[2] + hi[2]);
    size_t bi = 0;
    float bd = INFINITY;
    for (size_t i = 0; i < n; ++i) {
        const float dx = Pf[3 * i] - cx, dy = Pf[3 * i + 1] - cy, dz = Pf[3 * i + 2] - cz;
        const float d = dx * dx + dy * dy + dz * dz;
        if (d < bd) { bd = d; bi = i; }
    }
    for (int k = 0; k < 3; ++k) w.put(Pf[3 * bi + k]);
    return bytes;
}

bool bad_object(const int64_t* voff, const uint32_t* faces, const int64_t* foff, long o) {
    const int64_t n = voff[o + 1] - voff[o], m = foff[o + 1] - foff[o];
    if (n <= 0 || m <= 0) return true;
    for (int64_t f = foff[o]; f < foff[o + 1]; ++f) {
        const uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        if (a >= n || b >= n || c >= n || a == b || b == c || a == c) return true;
    }
    return false;
}

}  // namespace

extern "C" {

// RAW tile (zero bounds) of n_objects meshes: vertices[3 vert_off[o] ..) and
// faces[3 face_off[o] ..) (indices local to the object).  Call with out = null
// for the size.  threads <= 0: hardware concurrency.
long tdo_raw_from_meshes(const float* vertices, const int64_t* vert_off, const uint32_t* faces,
                         const int64_t* face_off, long n_objects, int voxel_size, uint8_t* out, size_t cap,
                         size_t* len, int threads) {
    if (voxel_size <= 0 || n_objects < 0) return -1;
    for (long o = 0; o < n_objects; ++o)
        if (bad_object(vert_off, faces, face_off, o)) return -1 - o;
    std::vector<size_t> sz(n_objects);
    const int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    auto run = [&](bool write, const std::vector<size_t>& pos) {
        std::vector<std::thread> ts;
        for (int t = 0; t < T; ++t)
            ts.emplace_back([&, t]() {
                for (long o = t; o < n_objects; o += T) {
                    const size_t s = prepare(vertices + 3 * vert_off[o], (size_t)(vert_off[o + 1] - vert_off[o]),
                                             faces + 3 * face_off[o], (size_t)(face_off[o + 1] - face_off[o]),
                                             voxel_size, write ? out + pos[o] : nullptr);
                    if (!write) sz[o] = s;
                }
            });
        for (auto& x : ts) x.join();
    };
    run(false, {});
    std::vector<size_t> pos(n_objects);
    size_t total = 1;
    for (long o = 0; o < n_objects; ++o) {
        pos[o] = total;
        total += sz[o];
    }
    if (len) *len = total;
    if (!out) return 0;
    if (cap < total) return -1;
    out[0] = 1;
    run(true, pos);
    return 0;
}

}  // extern "C"
