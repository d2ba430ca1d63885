// result.h -- the join result behind the opaque tdp_result of the C ABI
// (rows sorted by query id, then result id).
#pragma once
#include <vector>

struct tdp_result {
    std::vector<int> q, t;
    std::vector<float> d;
    std::vector<double> d64;  // exact LOD-100 distances (params.exact_distances)
};
