// candidates_capi.cpp -- C ABI of the object-level candidate generation.
#include <climits>
#include <cstring>

#include "index/candidates.h"
#include "tdp.h"

extern "C" long tdp_candidates(const float* box1, const float* xf1, long n1, const float* box2, const float* xf2,
                               long n2, int self_join, int is_knn, int knn, float within, int64_t* off, int32_t* ids,
                               long cap) {
    if (!box1 || !xf1 || !box2 || !xf2 || !off || n1 < 0 || n2 < 0 || (is_knn == 1 && knn < 1) || is_knn < 0 ||
        is_knn > 2)
        return LONG_MIN;
    // is_knn: 1 kNN, 0 within, 2 intersect (strict box overlap, ordered by id)
    tdp::CandidateQuery q{box1, xf1, n1, box2, xf2, n2, self_join != 0, is_knn == 1, knn, within, 0};
    q.strict_overlap = is_knn == 2;
    std::vector<int64_t> o;
    std::vector<int32_t> i;
    tdp::generate_candidates(q, o, i);
    std::memcpy(off, o.data(), o.size() * sizeof(int64_t));
    if ((long)i.size() > cap || !ids) return -(long)i.size();
    std::memcpy(ids, i.data(), i.size() * sizeof(int32_t));
    return (long)i.size();
}
