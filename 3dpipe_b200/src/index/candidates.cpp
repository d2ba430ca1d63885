// candidates.cpp -- grid-based object candidate generation (see candidates.h).
#include "index/candidates.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <queue>
#include <thread>

namespace tdp {

float box_gap(const float* a, const float* b) {
    // aab::distance (reference src/spatial/himesh_box.cpp:149-168), mindist part,
    // with a = the indexed object, b = the query box
    float m = 0.f;
    for (int i = 0; i < 3; ++i) {
        float t1 = a[i] - b[3 + i];
        float t2 = a[3 + i] - b[i];
        if (t2 < 0.f)
            m += t2 * t2;
        else if (t1 > 0.f)
            m += t1 * t1;
    }
    return std::sqrt(m);
}

float point_dist(const float* a, const float* b) {
    // octree.cpp:268-272: distance between the two objects' transform points
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

float pick_cell(const float* box, long n) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    std::vector<float> ext;
    ext.reserve(n);
    for (long i = 0; i < n; ++i) {
        float e = 0;
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], box[6 * i + k]);
            hi[k] = std::max(hi[k], box[6 * i + 3 + k]);
            e = std::max(e, box[6 * i + 3 + k] - box[6 * i + k]);
        }
        ext.push_back(e);
    }
    std::nth_element(ext.begin(), ext.begin() + ext.size() / 2, ext.end());
    double vol = 1;
    for (int k = 0; k < 3; ++k) vol *= std::max(1e-3f, hi[k] - lo[k]);
    float dens = (float)std::cbrt(vol / std::max<long>(n, 1));
    return std::max({ext[ext.size() / 2], dens, 1e-3f});
}

void generate_candidates(const CandidateQuery& q, std::vector<int64_t>& off, std::vector<int32_t>& ids) {
    off.assign(q.n1 + 1, 0);
    ids.clear();
    if (q.n1 <= 0) return;
    const float cell = pick_cell(q.box2, q.n2);
    CellGrid boxes, points;
    boxes.build(q.box2, q.n2, 6, 3, cell);
    if (q.is_knn || q.obj_knn) points.build(q.xf2, q.n2, 3, 0, cell);

    const int threads = q.threads > 0 ? q.threads : (int)std::max(1u, std::thread::hardware_concurrency());
    const long chunk = 256;
    const long nchunks = (q.n1 + chunk - 1) / chunk;
    std::vector<std::vector<int32_t>> part_ids(nchunks);
    std::vector<std::vector<int64_t>> part_cnt(nchunks);
    std::atomic<long> next{0};

    auto worker = [&]() {
        std::vector<int> stamp(q.n2, -1);
        std::vector<std::pair<float, int32_t>> found;
        for (long c; (c = next.fetch_add(1)) < nchunks;) {
            auto& out = part_ids[c];
            auto& cnts = part_cnt[c];
            for (long i = c * chunk; i < std::min(q.n1, (c + 1) * chunk); ++i) {
                const float* qb = q.box1 + 6 * i;
                const float* qx = q.xf1 + 3 * i;
                found.clear();
                if (i < q.q_begin || (q.q_end >= 0 && i >= q.q_end)) {
                    cnts.push_back(0);
                    continue;
                }
                const bool is_knn = q.obj_knn ? q.obj_knn[i] > 0 : q.is_knn;
                const float within = q.obj_knn ? q.obj_within[i] : q.within;
                if (!is_knn) {
                    const float r = within;
                    int x0 = boxes.ci(qb[0] - r, 0), x1 = boxes.ci(qb[3] + r, 0);
                    int y0 = boxes.ci(qb[1] - r, 1), y1 = boxes.ci(qb[4] + r, 1);
                    int z0 = boxes.ci(qb[2] - r, 2), z1 = boxes.ci(qb[5] + r, 2);
                    for (int x = x0; x <= x1; ++x)
                        for (int y = y0; y <= y1; ++y)
                            for (int z = z0; z <= z1; ++z) {
                                size_t cc = boxes.id(x, y, z);
                                for (int64_t k = boxes.start[cc]; k < boxes.start[cc + 1]; ++k) {
                                    int32_t o = boxes.items[k];
                                    if (stamp[o] == (int)i) continue;
                                    stamp[o] = (int)i;
                                    if (q.self_join && o == i) continue;
                                    const float* ob = q.box2 + 6 * o;
                                    const bool hit =
                                        q.strict_overlap
                                            ? !(ob[0] >= qb[3] || ob[3] <= qb[0] || ob[1] >= qb[4] || ob[4] <= qb[1] ||
                                                ob[2] >= qb[5] || ob[5] <= qb[2])
                                            : box_gap(ob, qb) <= within;
                                    if (hit) found.push_back({0.f, o});
                                }
                            }
                    std::sort(found.begin(), found.end(), [](auto& a, auto& b) { return a.second < b.second; });
                } else {
                    // 1) the K smallest transform distances (ring search on the point grid)
                    const int K = q.obj_knn ? q.obj_knn[i] : q.knn;
                    std::priority_queue<std::pair<float, int32_t>> heap;  // max-heap of (dist, id)
                    int cx = points.ci(qx[0], 0), cy = points.ci(qx[1], 1), cz = points.ci(qx[2], 2);
                    int maxr = std::max({points.n[0], points.n[1], points.n[2]});
                    for (int r = 0; r <= maxr; ++r) {
                        for (int x = cx - r; x <= cx + r; ++x)
                            for (int y = cy - r; y <= cy + r; ++y)
                                for (int z = cz - r; z <= cz + r; ++z) {
                                    if (std::max({std::abs(x - cx), std::abs(y - cy), std::abs(z - cz)}) != r) continue;
                                    if (x < 0 || y < 0 || z < 0 || x >= points.n[0] || y >= points.n[1] || z >= points.n[2]) continue;
                                    size_t cc = points.id(x, y, z);
                                    for (int64_t k = points.start[cc]; k < points.start[cc + 1]; ++k) {
                                        int32_t o = points.items[k];
                                        if (q.self_join && o == i) continue;
                                        std::pair<float, int32_t> e = {point_dist(qx, q.xf2 + 3 * o), o};
                                        if ((int)heap.size() < K) heap.push(e);
                                        else if (e < heap.top()) { heap.pop(); heap.push(e); }
                                    }
                                }
                        if ((int)heap.size() == K && heap.top().first < (float)r * points.cell - points.slack) break;
                    }
                    const float maxk = (int)heap.size() == K ? heap.top().first : INFINITY;
                    std::vector<int32_t> topk;
                    while (!heap.empty()) { topk.push_back(heap.top().second); heap.pop(); }
                    for (int32_t o : topk) stamp[o] = (int)i;
                    for (int32_t o : topk) found.push_back({point_dist(qx, q.xf2 + 3 * o), o});
                    // 2) every object whose box gap is below the K-th distance
                    const float r = std::isfinite(maxk) ? maxk : 3e38f;
                    int x0 = boxes.ci(qb[0] - r, 0), x1 = boxes.ci(qb[3] + r, 0);
                    int y0 = boxes.ci(qb[1] - r, 1), y1 = boxes.ci(qb[4] + r, 1);
                    int z0 = boxes.ci(qb[2] - r, 2), z1 = boxes.ci(qb[5] + r, 2);
                    for (int x = x0; x <= x1; ++x)
                        for (int y = y0; y <= y1; ++y)
                            for (int z = z0; z <= z1; ++z) {
                                size_t cc = boxes.id(x, y, z);
                                for (int64_t k = boxes.start[cc]; k < boxes.start[cc + 1]; ++k) {
                                    int32_t o = boxes.items[k];
                                    if (stamp[o] == (int)i) continue;
                                    stamp[o] = (int)i;
                                    if (q.self_join && o == i) continue;
                                    if (box_gap(q.box2 + 6 * o, qb) < maxk) found.push_back({point_dist(qx, q.xf2 + 3 * o), o});
                                }
                            }
                    std::sort(found.begin(), found.end());
                }
                for (auto& f : found) out.push_back(f.second);
                cnts.push_back((int64_t)found.size());
            }
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t) ts.emplace_back(worker);
    for (auto& t : ts) t.join();
    long i = 0;
    for (long c = 0; c < nchunks; ++c) {
        for (int64_t n : part_cnt[c]) {
            off[i + 1] = off[i] + n;
            ++i;
        }
        ids.insert(ids.end(), part_ids[c].begin(), part_ids[c].end());
    }
}

}  // namespace tdp
