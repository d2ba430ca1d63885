// oracle/ref_join.cpp -- TEST INFRASTRUCTURE and the timed CPU baseline only.
//
// Runs the reference's join on the CPU with the reference's own compute code,
// compiled from source into oracle/_ref/libtdp_ref.so:
//   * candidates: the reference octree (tdr_candidates in ref_shim.cpp:
//     build_octree leaf 10 + query_knn_fast / query_within);
//   * refine: the reference's FP32 MeshDist (src/geometry/computing_cpu.cpp:441-481).
// The control flow between those calls is restated from the reference's GPU
// join path, which is what `tdbase join -g` runs (the reference has no complete
// CPU-only join: src/join/KNNJoin.cpp:1530 and WithinJoin.cpp:648 call GPU
// filters unconditionally):
//   filter bounds            voxel_dist_core             computing_gpu.cu:1606-1631
//   kNN rank + confirm cap   evaluate_knn_kernel          computing_gpu.cu:105-151,
//                            evaluate_candidate_lists_gpu KNNJoin.cpp:133-202
//   within classification    WithinJoin.cpp:164-252, :769-792
//   voxel-pair compaction    computing_gpu.cu:2604-2812
//   bound update / eviction  KNNJoin.cpp:1668-1705, SpatialJoin.cpp:48-69
// Threads: one std::thread per host core over object pairs (the reference
// parallelises the same loops with OpenMP and pthreads).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "geometry.h"
#include "rawdt.hpp"

extern "C" long tdr_candidates_sel(const float* box1, const float* xf1, long n1, const float* box2,
                                   const float* xf2, long n2, int self_join, int knn, float within, int is_knn,
                                   const int* qmap, long* off, int* ids, long cap);

namespace {

using oracle::RObject;
using oracle::RVoxel;

void vdist(const RVoxel& a, const RVoxel& b, float& mn, float& mx) {
    float m = 0.f, M = 0.f;
    for (int i = 0; i < 3; ++i) {
        float t1 = a.low[i] - b.high[i], t2 = a.high[i] - b.low[i];
        if (t2 < 0.f) m += t2 * t2;
        else if (t1 > 0.f) m += t1 * t1;
        float dc = a.core[i] - b.core[i];
        M += dc * dc;
    }
    mn = std::sqrt(m);
    mx = std::sqrt(M);
}

struct VPair {
    int a, b;
    float mn, mx;
    bool alive = true;
    bool upd = false;
};

struct Pair {
    int q, t;
    float mn, mx;
    int stat = 0;  // 0 undecided, 1 reported, 2 dropped
    std::vector<VPair> vps;
};

template <typename Fn>
void par(long n, int threads, Fn fn) {
    std::atomic<long> next{0};
    std::vector<std::thread> ts;
    for (int i = 0; i < threads; ++i)
        ts.emplace_back([&]() {
            for (long k; (k = next.fetch_add(1)) < n;) fn(k);
        });
    for (auto& t : ts) t.join();
}

void knn_rank(std::vector<Pair>& P, long b, long e, int K, int& conf) {
    if (conf < K) {
        const int left = K - conf;
        std::vector<int> st(e - b, 0);
        for (long i = b; i < e; ++i) {
            if (P[i].stat) continue;
            int sure = 0, maybe = 0;
            for (long j = b; j < e; ++j) {
                if (j == i || P[j].stat) continue;
                if (P[i].mn >= P[j].mx) ++sure;
                if (!(P[i].mx <= P[j].mn)) ++maybe;
            }
            st[i - b] = maybe < left ? 1 : (sure >= left ? 2 : 0);
        }
        for (long i = b; i < e && conf < K; ++i) {
            if (P[i].stat) continue;
            if (st[i - b] == 1) { P[i].stat = 1; ++conf; }
            else if (st[i - b] == 2) P[i].stat = 2;
        }
    }
    if (conf >= K)
        for (long i = b; i < e; ++i)
            if (!P[i].stat) P[i].stat = 2;
}

// The join for the query objects qsel (ids into tile 1); when qsel is empty,
// for the first max_queries objects of tile 1, or all of them when
// max_queries <= 0.  Results are (tile-1 id, tile-2 id) pairs.
//
// cap_rel >= 0 (within joins at Hausdorff level 2 only) replays a cap on the
// LODs before the last: at each such LOD a pair's cap is C = max(tau, the
// smallest upper bound vmx of the voxel pairs this LOD refines) * (1 +
// cap_rel) + cap_rel, above the pair's minmax after the LOD (vmx is a running
// minimum); a voxel pair whose Hausdorff lower bound comes out above C keeps
// its previous vmn and vmx.  cap_stats (2 doubles): such voxel-pair refines
// and their triangle pairs.
long join_impl(const uint8_t* b1, size_t l1, const uint8_t* b2, size_t l2, int self_join, int is_knn, int knn,
               float tau, const int* lods, int nlods, int level, int threads, long max_queries, std::vector<int> qsel,
               int* oq, int* ot, long cap, double* stats, float cap_rel = -1.f, double* cap_stats = nullptr) {
    auto t0 = std::chrono::steady_clock::now();
    std::vector<RObject> T1 = oracle::read_tile(b1, l1);
    std::vector<RObject> T2 = self_join ? std::vector<RObject>() : oracle::read_tile(b2, l2);
    const std::vector<RObject>& S = self_join ? T1 : T2;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (qsel.empty()) {
        long n = (long)T1.size();
        if (max_queries > 0 && max_queries < n) n = max_queries;
        for (long i = 0; i < n; ++i) qsel.push_back((int)i);
    }
    for (int q : qsel)
        if (q < 0 || q >= (long)T1.size()) return 0;
    long n1 = (long)qsel.size(), n2 = (long)S.size();
    std::vector<float> box1(6 * n1), xf1(3 * n1), box2(6 * n2), xf2(3 * n2);
    for (long i = 0; i < n1; ++i) {
        std::memcpy(&box1[6 * i], T1[qsel[i]].box, 24);
        std::memcpy(&xf1[3 * i], T1[qsel[i]].transform, 12);
    }
    for (long i = 0; i < n2; ++i) { std::memcpy(&box2[6 * i], S[i].box, 24); std::memcpy(&xf2[3 * i], S[i].transform, 12); }
    // candidates from the reference octree for the chosen query objects
    std::vector<long> off(n1 + 1);
    std::vector<int> ids;
    long capc = std::max<long>(1024, n1 * 64);
    for (;;) {
        ids.assign(capc, 0);
        long tot = tdr_candidates_sel(box1.data(), xf1.data(), n1, box2.data(), xf2.data(), n2, self_join, knn, tau,
                                      is_knn, qsel.data(), off.data(), ids.data(), capc);
        if (tot >= 0) { ids.resize(tot); break; }
        capc *= 4;
    }
    std::vector<Pair> P;
    for (long q = 0; q < n1; ++q)
        for (long k = off[q]; k < off[q + 1]; ++k) { Pair p; p.q = qsel[q]; p.t = ids[k]; P.push_back(p); }
    std::vector<long> qoff(off.begin(), off.begin() + n1 + 1);
    std::vector<int> conf(n1, 0);
    // filter
    par((long)P.size(), threads, [&](long i) {
        Pair& p = P[i];
        float mn = FLT_MAX, mx = FLT_MAX;
        for (auto& a : T1[p.q].vox)
            for (auto& b : S[p.t].vox) {
                float m, M;
                vdist(a, b, m, M);
                mn = std::min(mn, m);
                mx = std::min(mx, M);
            }
        p.mn = mn;
        p.mx = mx;
        if (!is_knn) {
            if (mn > tau) p.stat = 2;
            else if (mx <= tau) p.stat = 1;
        }
    });
    if (is_knn) par(n1, threads, [&](long q) { knn_rank(P, qoff[q], qoff[q + 1], knn, conf[q]); });
    par((long)P.size(), threads, [&](long i) {
        Pair& p = P[i];
        if (p.stat) return;
        const auto& A = T1[p.q].vox;
        const auto& B = S[p.t].vox;
        for (int a = 0; a < (int)A.size(); ++a)
            for (int b = 0; b < (int)B.size(); ++b) {
                float m, M;
                vdist(A[a], B[b], m, M);
                if (m <= p.mx && (is_knn || m <= tau)) p.vps.push_back({a, b, m, M});
            }
    });
    // LOD loop
    std::vector<int> L(lods, lods + nlods);
    if (L.empty()) L = {20, 40, 60, 80, 100};
    std::sort(L.begin(), L.end());
    L.erase(std::unique(L.begin(), L.end()), L.end());
    std::atomic<long long> tri_pairs{0}, vp_refined{0}, capped_vp{0}, capped_tp{0};
    for (size_t k = 0; k < L.size(); ++k) {
        const int li = L[k] / 20 - 1;
        const bool highest = k + 1 == L.size();
        const bool capping = cap_rel >= 0.f && !is_knn && level == 2 && !highest;
        par((long)P.size(), threads, [&](long i) {
            Pair& p = P[i];
            if (p.stat) return;
            std::vector<float> ta, ha, tb, hb;
            double minmax = DBL_MAX;
            long long tp = 0, nv = 0, cvp = 0, ctp = 0;
            float C = FLT_MAX;
            if (capping) {
                float base = FLT_MAX;
                for (auto& v : p.vps)
                    if (v.alive && T1[p.q].vox[v.a].cnt[li] && S[p.t].vox[v.b].cnt[li]) base = std::min(base, v.mx);
                if (base < FLT_MAX) C = std::max(tau, base) * (1.f + cap_rel) + cap_rel;
            }
            for (auto& v : p.vps) {
                v.upd = false;
                if (!v.alive) continue;
                const RVoxel& A = T1[p.q].vox[v.a];
                const RVoxel& B = S[p.t].vox[v.b];
                if (!A.cnt[li] || !B.cnt[li]) continue;
                T1[p.q].tris(v.a, li, ta, ha);
                S[p.t].tris(v.b, li, tb, hb);
                tdbase::result_container r =
                    tdbase::MeshDist(ta.data(), tb.data(), A.cnt[li], B.cnt[li], ha.data(), hb.data());
                tp += (long long)(A.cnt[li] * B.cnt[li]);
                ++nv;
                if (highest) { v.mn = r.distance; v.mx = r.distance; }
                else if (capping && r.min_dist > C) { ++cvp; ctp += (long long)(A.cnt[li] * B.cnt[li]); }
                else if (level == 2) { v.mn = std::min(v.mn, r.min_dist); v.mx = std::min(v.mx, r.max_dist); }
                else if (level == 1) {
                    v.mn = std::min(v.mn, r.distance - T1[p.q].hd[li] - S[p.t].hd[li]);
                    v.mx = std::min(v.mx, r.distance + T1[p.q].phd[li] + S[p.t].phd[li]);
                } else v.mx = std::min(v.mx, r.distance);
                v.upd = true;
                minmax = std::min(minmax, (double)v.mx);
            }
            float mind = FLT_MAX;
            for (auto& v : p.vps)
                if (v.alive) {
                    mind = std::min(mind, v.mn);
                    if (v.mn > minmax) v.alive = false;
                }
            p.mn = mind;
            p.mx = (float)minmax;
            if (!is_knn) {
                if (p.mx <= tau) p.stat = 1;
                else if (p.mn > tau) p.stat = 2;
            }
            tri_pairs += tp;
            vp_refined += nv;
            capped_vp += cvp;
            capped_tp += ctp;
        });
        if (is_knn) par(n1, threads, [&](long q) { knn_rank(P, qoff[q], qoff[q + 1], knn, conf[q]); });
        long und = 0;
        for (auto& p : P) und += p.stat == 0;
        if (!und) break;
    }
    long n = 0;
    for (auto& p : P)
        if (p.stat == 1) {
            if (n < cap) { oq[n] = p.q; ot[n] = p.t; }
            ++n;
        }
    if (stats) {
        stats[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        stats[1] = (double)tri_pairs.load();
        stats[2] = (double)vp_refined.load();
        stats[3] = (double)P.size();
    }
    if (cap_stats) {
        cap_stats[0] = (double)capped_vp.load();
        cap_stats[1] = (double)capped_tp.load();
    }
    return n <= cap ? n : -n;
}

}  // namespace

// stats (optional, 4 doubles): seconds, triangle pairs refined, voxel pairs refined, candidates.
// max_queries > 0 joins only the first max_queries objects of tile 1.
extern "C" long tdr_join(const uint8_t* b1, size_t l1, const uint8_t* b2, size_t l2, int self_join, int is_knn,
                         int knn, float tau, const int* lods, int nlods, int level, int threads, long max_queries,
                         int* oq, int* ot, long cap, double* stats) {
    return join_impl(b1, l1, b2, l2, self_join, is_knn, knn, tau, lods, nlods, level, threads, max_queries, {}, oq, ot,
                     cap, stats);
}

// The same join for the query objects qids[0..nq) of tile 1 (a sample of
// queries: per-object candidate lists never mix query objects, so each
// query's result is the one the whole join gives it).  Ids must be in range.
extern "C" long tdr_join_sel(const uint8_t* b1, size_t l1, const uint8_t* b2, size_t l2, int self_join, int is_knn,
                             int knn, float tau, const int* lods, int nlods, int level, int threads, const int* qids,
                             long nq, int* oq, int* ot, long cap, double* stats) {
    if (nq <= 0) return 0;
    return join_impl(b1, l1, b2, l2, self_join, is_knn, knn, tau, lods, nlods, level, threads, 0,
                     std::vector<int>(qids, qids + nq), oq, ot, cap, stats);
}

// tdr_join with the cap of join_impl replayed (cap_rel >= 0); cap_stats as there.
extern "C" long tdr_join_capped(const uint8_t* b1, size_t l1, const uint8_t* b2, size_t l2, int self_join,
                                int is_knn, int knn, float tau, const int* lods, int nlods, int level, int threads,
                                float cap_rel, int* oq, int* ot, long cap, double* stats, double* cap_stats) {
    return join_impl(b1, l1, b2, l2, self_join, is_knn, knn, tau, lods, nlods, level, threads, 0, {}, oq, ot, cap,
                     stats, cap_rel, cap_stats);
}
