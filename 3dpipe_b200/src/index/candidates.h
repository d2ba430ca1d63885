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
};

// off: [n1+1] CSR offsets into ids.
void generate_candidates(const CandidateQuery& q, std::vector<int64_t>& off, std::vector<int32_t>& ids);

// The reference's float formulas (exposed for tests).
float box_gap(const float* a, const float* b);
float point_dist(const float* a, const float* b);

}  // namespace tdp
