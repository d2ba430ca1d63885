// candidates.h -- object-level candidate generation (the first filter level).
//
// Restates what the reference's octree queries return (src/index/octree.cpp:120-154,
// :215-291, :293-330; called at src/join/KNNJoin.cpp:553-573 and
// src/join/WithinJoin.cpp:80-97), with a uniform grid instead of an octree:
//   kNN (query_knn_fast): with maxdist(o) = |transform(q) - transform(o)| and
//     mindist(o) = gap between the two object boxes (aab::distance,
//     src/spatial/himesh_box.cpp:149-168), the candidates are the K objects
//     with the smallest maxdist plus every object with mindist < the K-th
//     smallest maxdist; ordered by (maxdist, id).
//   within (query_within): every object with mindist <= tau; ordered by id.
// In a self-join the query object itself is excluded (octree.cpp:253, :299).
// All distances use the reference's float arithmetic so membership at
// boundaries matches.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace tdp {

struct CandidateQuery {
    const float* box1;  // 6 per query object (low xyz, high xyz)
    const float* xf1;   // 3 per query object
    long n1;
    const float* box2;
    const float* xf2;
    long n2;
    bool self_join;
    bool is_knn;
    int knn;
    float within;
    int threads;  // 0 = hardware concurrency
    // optional per query object query (a batch of different requests):
    // obj_knn[i] = K (> 0, kNN) or 0 (within, distance obj_within[i])
    const int* obj_knn = nullptr;
    const float* obj_within = nullptr;
    // intersect query: candidates are objects whose boxes overlap strictly
    bool strict_overlap = false;
    // only query objects [q_begin, q_end) get candidates (q_end < 0: to n1);
    // the others get empty lists
    long q_begin = 0;
    long q_end = -1;
};

// off: [n1+1] CSR offsets into ids.
void generate_candidates(const CandidateQuery& q, std::vector<int64_t>& off, std::vector<int32_t>& ids);

// Uniform grid over object boxes (a point grid passes lo == hi): CSR of the
// objects overlapping each cell.  The cell is enlarged until there are at most
// about 8 cells per object.
struct CellGrid {
    float lo[3] = {0, 0, 0};
    float cell = 1.f;
    int n[3] = {1, 1, 1};
    // Bound on how far float rounding in ci() can move a point across a cell
    // face: a ring search stops only when its K-th distance is below the ring
    // radius by more than this, so a point assigned to a neighbouring cell by
    // rounding, or one at exactly the ring radius, is never missed.
    float slack = 0.f;
    std::vector<int64_t> start;  // CSR over cells
    std::vector<int32_t> items;

    int ci(float v, int k) const {
        long c = (long)std::floor((v - lo[k]) / cell);
        return (int)std::min<long>(std::max<long>(c, 0), n[k] - 1);
    }
    size_t id(int x, int y, int z) const { return ((size_t)x * n[1] + y) * n[2] + z; }

    // boxes: 6 floats per object (a point grid passes lo == hi)
    void build(const float* boxes, long count, int stride_lo, int stride_hi, float cell_) {
        cell = cell_;
        float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        lo[0] = lo[1] = lo[2] = INFINITY;
        for (long i = 0; i < count; ++i)
            for (int k = 0; k < 3; ++k) {
                lo[k] = std::min(lo[k], boxes[i * stride_lo + k]);
                hi[k] = std::max(hi[k], boxes[i * stride_lo + stride_hi + k]);
            }
        // keep the number of cells bounded (about 8 per object)
        const double max_cells = std::max(4096.0, 8.0 * (double)count);
        auto cells_for = [&](float c) {
            double p = 1;
            for (int k = 0; k < 3; ++k) p *= std::ceil((hi[k] - lo[k]) / c) + 1;
            return p;
        };
        while (cells_for(cell) > max_cells) cell *= 1.25f;
        for (int k = 0; k < 3; ++k) n[k] = std::max(1, (int)std::ceil((hi[k] - lo[k]) / cell) + 1);
        slack = 0.f;
        for (int k = 0; k < 3; ++k) slack = std::max(slack, std::fabs(lo[k]) + (float)n[k] * cell);
        slack *= 1e-5f;
        std::vector<int64_t> cnt(id(n[0] - 1, n[1] - 1, n[2] - 1) + 2, 0);
        auto each = [&](long i, auto fn) {
            const float* b = boxes + i * stride_lo;
            int x0 = ci(b[0], 0), x1 = ci(b[stride_hi + 0], 0), y0 = ci(b[1], 1), y1 = ci(b[stride_hi + 1], 1);
            int z0 = ci(b[2], 2), z1 = ci(b[stride_hi + 2], 2);
            for (int x = x0; x <= x1; ++x)
                for (int y = y0; y <= y1; ++y)
                    for (int z = z0; z <= z1; ++z) fn(id(x, y, z));
        };
        for (long i = 0; i < count; ++i) each(i, [&](size_t c) { cnt[c + 1]++; });
        for (size_t c = 1; c < cnt.size(); ++c) cnt[c] += cnt[c - 1];
        start = cnt;
        items.resize(start.back());
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (long i = 0; i < count; ++i) each(i, [&](size_t c) { items[fill[c]++] = (int32_t)i; });
    }
};

// cell size for a set of boxes: the median box extent or the mean spacing
float pick_cell(const float* box, long n);

// The reference's float formulas (exposed for tests).
float box_gap(const float* a, const float* b);
float point_dist(const float* a, const float* b);

}  // namespace tdp
