// partition.cpp -- splitting a join's query objects over N GPUs by estimated
// work (tdp_partition_queries / tdp_raw_partition, include/tdp.h).
//
// The reference runs on one GPU (src/geometry/cuda_common.cu:20), but its
// join already treats query objects independently: every query object has its
// own candidate list (src/join/KNNJoin.cpp:552-600,
// src/join/WithinJoin.cpp:79-99) and its own filter and LOD loop over it.
// So a join over N GPUs gives each GPU a contiguous range of query objects and
// the whole tile 2; the ranges are cut where the prefix sum of the per-object
// work estimate crosses s/N of the total.  The estimate is what the filter
// costs and what the refine grows with: the voxel pairs of the object's
// candidates, n_voxels(query) x n_voxels(candidate), plus one per object.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "index/candidates.h"
#include "storage/dt_format.h"
#include "tdp.h"

namespace tdp {
namespace {

int partition_impl(const CandidateQuery& cq, const uint32_t* nvox1, const uint32_t* nvox2, int n_shards,
                   long* bounds, double* work) {
    const long n1 = cq.n1;
    std::vector<int64_t> off;
    std::vector<int32_t> ids;
    generate_candidates(cq, off, ids);
    std::vector<double> prefix(n1 + 1, 0.0);
    for (long i = 0; i < n1; ++i) {
        double w = 1.0;
        for (int64_t k = off[i]; k < off[i + 1]; ++k) w += (double)nvox1[i] * (double)nvox2[ids[k]];
        prefix[i + 1] = prefix[i] + w;
    }
    const double total = prefix[n1];
    bounds[0] = 0;
    long cur = 0;
    for (int sh = 1; sh < n_shards; ++sh) {
        const double target = total * (double)sh / (double)n_shards;
        // first object boundary whose prefix reaches the target
        cur = std::max<long>(cur, std::lower_bound(prefix.begin(), prefix.end(), target) - prefix.begin());
        bounds[sh] = std::min(cur, n1);
    }
    bounds[n_shards] = n1;
    if (work)
        for (int sh = 0; sh < n_shards; ++sh) work[sh] = prefix[bounds[sh + 1]] - prefix[bounds[sh]];
    return TDP_OK;
}

std::vector<uint32_t> voxel_counts(const TileHost& h) {
    std::vector<uint32_t> n(h.n_obj);
    for (long i = 0; i < h.n_obj; ++i) n[i] = h.obj_vox_off[i + 1] - h.obj_vox_off[i];
    return n;
}

void put_err(char* err, size_t cap, const std::string& m) {
    if (err && cap) {
        std::strncpy(err, m.c_str(), cap - 1);
        err[cap - 1] = 0;
    }
}

}  // namespace
}  // namespace tdp

using namespace tdp;

extern "C" int tdp_partition_queries(const float* box1, const float* xf1, const uint32_t* nvox1, long n1,
                                     const float* box2, const float* xf2, const uint32_t* nvox2, long n2,
                                     int self_join, int is_knn, int knn, float within, int n_shards, long* bounds,
                                     double* work) {
    if (n1 < 0 || n2 < 0 || n_shards < 1 || !bounds) return TDP_ERR_ARG;
    if (n1 > 0 && (!box1 || !xf1 || !nvox1)) return TDP_ERR_ARG;
    if (n2 > 0 && (!box2 || !xf2 || !nvox2)) return TDP_ERR_ARG;
    if (is_knn < 0 || is_knn > 2 || (is_knn == 1 && knn < 1)) return TDP_ERR_ARG;
    if (self_join && n1 != n2) return TDP_ERR_ARG;
    CandidateQuery cq{box1, xf1, n1, box2, xf2, n2, self_join != 0, is_knn == 1, is_knn == 1 ? knn : 0, within, 0};
    cq.strict_overlap = is_knn == 2;
    return partition_impl(cq, nvox1, nvox2, n_shards, bounds, work);
}

extern "C" int tdp_raw_partition(const void* raw1, size_t len1, const void* raw2, size_t len2, int is_knn, int knn,
                                 float within, int n_shards, long* bounds, double* work, char* err, size_t err_cap) {
    if (!raw1 || n_shards < 1 || !bounds || is_knn < 0 || is_knn > 2 || (is_knn == 1 && knn < 1)) {
        put_err(err, err_cap, "bad arguments");
        return TDP_ERR_ARG;
    }
    TileHost h1, h2;
    std::string e;
    int rc = parse_raw_dt((const uint8_t*)raw1, len1, 0, h1, e);
    if (rc == TDP_OK && raw2) rc = parse_raw_dt((const uint8_t*)raw2, len2, 0, h2, e);
    if (rc != TDP_OK) {
        put_err(err, err_cap, e);
        return rc;
    }
    const bool self = raw2 == nullptr;
    const TileHost& t2 = self ? h1 : h2;
    const std::vector<uint32_t> n1v = voxel_counts(h1), n2v = self ? n1v : voxel_counts(h2);
    CandidateQuery cq{h1.obj_box.data(), h1.obj_xf.data(), h1.n_obj, t2.obj_box.data(), t2.obj_xf.data(), t2.n_obj,
                      self, is_knn == 1, is_knn == 1 ? knn : 0, within, 0};
    cq.strict_overlap = is_knn == 2;
    return partition_impl(cq, n1v.data(), n2v.data(), n_shards, bounds, work);
}
