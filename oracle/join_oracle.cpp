// oracle/join_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the FP64 exact join.
//
// Ground truth for the joins the reference answers (kNN: src/join/KNNJoin.cpp,
// within: src/join/WithinJoin.cpp), computed without any of the filter's
// bounds: the exact LOD-100 distance between two objects is the minimum FP64
// triangle distance (tdo_tri_dist, tridist.c) over all triangle pairs, found by
// branch and bound over voxel pairs in increasing box-gap order (a voxel box
// covers every triangle of its voxel, so the gap is a lower bound).
//   kNN:    the K smallest exact distances per query object (ties by id);
//   within: every object at exact distance <= tau.
// In a self-join the query object is excluded.  Every evaluated (query, object)
// pair is returned with its exact distance and whether it is a result, so tests
// can also check that the seeded inputs have no near-ties.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <queue>
#include <thread>
#include <vector>

#include "oracle.h"
#include "rawdt.hpp"

using oracle::RObject;

namespace {

double box_gap(const float* alo, const float* ahi, const float* blo, const float* bhi) {
    double s = 0;
    for (int k = 0; k < 3; ++k) {
        double g = std::max({(double)alo[k] - bhi[k], (double)blo[k] - ahi[k], 0.0});
        s += g * g;
    }
    return std::sqrt(s);
}

struct DTri {
    double v[9];
    double c[3];
    double r;
};

void to_dtris(const std::vector<float>& t, std::vector<DTri>& out) {
    const size_t n = t.size() / 9;
    out.resize(n);
    for (size_t i = 0; i < n; ++i) {
        DTri& d = out[i];
        for (int k = 0; k < 9; ++k) d.v[k] = t[9 * i + k];
        for (int k = 0; k < 3; ++k) d.c[k] = (d.v[k] + d.v[3 + k] + d.v[6 + k]) / 3.0;
        double r2 = 0;
        for (int j = 0; j < 3; ++j) {
            double dx = d.v[3 * j] - d.c[0], dy = d.v[3 * j + 1] - d.c[1], dz = d.v[3 * j + 2] - d.c[2];
            r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
        }
        d.r = std::sqrt(r2);
    }
}

// exact LOD-100 distance between two objects
double object_distance(const RObject& A, const RObject& B) {
    struct VP {
        double gap;
        int a, b;
    };
    std::vector<VP> vps;
    vps.reserve(A.vox.size() * B.vox.size());
    for (int a = 0; a < (int)A.vox.size(); ++a)
        for (int b = 0; b < (int)B.vox.size(); ++b)
            vps.push_back({box_gap(A.vox[a].low, A.vox[a].high, B.vox[b].low, B.vox[b].high), a, b});
    std::sort(vps.begin(), vps.end(), [](const VP& x, const VP& y) { return x.gap < y.gap; });
    double best = INFINITY;
    std::vector<float> ta, ha, tb, hb;
    std::vector<DTri> da, db;
    int cached_a = -1, cached_b = -1;
    for (const VP& vp : vps) {
        if (vp.gap > best) break;
        if (vp.a != cached_a) { A.tris(vp.a, 4, ta, ha); to_dtris(ta, da); cached_a = vp.a; }
        if (vp.b != cached_b) { B.tris(vp.b, 4, tb, hb); to_dtris(tb, db); cached_b = vp.b; }
        for (const DTri& x : da)
            for (const DTri& y : db) {
                double dx = x.c[0] - y.c[0], dy = x.c[1] - y.c[1], dz = x.c[2] - y.c[2];
                double lb = std::sqrt(dx * dx + dy * dy + dz * dz) - x.r - y.r;
                if (lb > best) continue;
                double d = tdo_tri_dist(x.v, y.v);
                if (d < best) best = d;
            }
    }
    return best;
}

struct Eval {
    int q, t;
    double d;
    int in;
};

}  // namespace

extern "C" long tdo_join_exact(const uint8_t* b1, size_t l1, const uint8_t* b2, size_t l2, int self_join, int is_knn,
                               int knn, double tau, int threads, int* oq, int* ot, double* od, int* oin, long cap) {
    std::vector<RObject> T1 = oracle::read_tile(b1, l1);
    std::vector<RObject> T2 = self_join ? std::vector<RObject>() : oracle::read_tile(b2, l2);
    const std::vector<RObject>& S = self_join ? T1 : T2;
    const long n1 = (long)T1.size();
    std::vector<std::vector<Eval>> per(n1);
    std::atomic<long> next{0};
    auto work = [&]() {
        for (long q; (q = next.fetch_add(1)) < n1;) {
            const RObject& Q = T1[q];
            std::vector<std::pair<double, int>> order;
            for (int t = 0; t < (int)S.size(); ++t) {
                if (self_join && t == q) continue;
                order.push_back({box_gap(Q.box, Q.box + 3, S[t].box, S[t].box + 3), t});
            }
            std::sort(order.begin(), order.end());
            auto& ev = per[q];
            if (is_knn) {
                std::priority_queue<std::pair<double, int>> best;  // max-heap of (D, id)
                for (auto& g : order) {
                    if ((int)best.size() == knn && g.first > best.top().first) break;
                    double D = object_distance(Q, S[g.second]);
                    ev.push_back({(int)q, g.second, D, 0});
                    std::pair<double, int> e = {D, g.second};
                    if ((int)best.size() < knn) best.push(e);
                    else if (e < best.top()) { best.pop(); best.push(e); }
                }
                std::vector<int> res;
                while (!best.empty()) { res.push_back(best.top().second); best.pop(); }
                for (auto& e : ev)
                    if (std::find(res.begin(), res.end(), e.t) != res.end()) e.in = 1;
            } else {
                for (auto& g : order) {
                    if (g.first > tau) break;
                    double D = object_distance(Q, S[g.second]);
                    ev.push_back({(int)q, g.second, D, D <= tau ? 1 : 0});
                }
            }
        }
    };
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> ts;
    for (int i = 0; i < nt; ++i) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    long total = 0;
    for (auto& v : per) total += (long)v.size();
    if (total > cap) return -total;
    long k = 0;
    for (auto& v : per)
        for (auto& e : v) {
            oq[k] = e.q;
            ot[k] = e.t;
            od[k] = e.d;
            oin[k] = e.in;
            ++k;
        }
    return total;
}
