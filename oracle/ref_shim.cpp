/*
 * oracle/ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A C-ABI shim around the reference's own CPU code, compiled unmodified from
 * the reference tree by oracle/Makefile into oracle/_ref/libtdp_ref.so:
 *   src/geometry/computing_cpu.cpp   TriDist, MeshDist  (FP32, the reference's CPU twin)
 *   src/geometry/TriInt.cpp          (linked only because MeshInt references it)
 *   src/index/octree.cpp             build_octree, query_knn_fast, query_within
 *   src/spatial/himesh_box.cpp       aab::distance and friends
 * This file is new code; it only adapts plain arrays to the reference's types
 * so the oracle and the CUDA path can be pinned against the reference itself.
 */
#include <algorithm>
#include <vector>
#include <utility>
#include <cstring>
#include <cstdint>
#include "aab.h"
#include "index.h"
#include "geometry.h"

using tdbase::range;
using tdbase::weighted_aab;
using tdbase::OctreeNode;

extern "C" {

float tdr_tri_dist(const float *S, const float *T) { return tdbase::TriDist(S, T); }

void tdr_tri_dist_batch(const float *S, const float *T, size_t n, float *out)
{
    for (size_t i = 0; i < n; ++i) out[i] = tdbase::TriDist(S + 9 * i, T + 9 * i);
}

/* MeshDist (computing_cpu.cpp:441-481): out = {distance, min_dist, max_dist} */
void tdr_mesh_dist(const float *d1, const float *d2, size_t n1, size_t n2,
                   const float *h1, const float *h2, float out[3])
{
    tdbase::result_container r = tdbase::MeshDist(d1, d2, n1, n2, h1, h2);
    out[0] = r.distance;
    out[1] = r.min_dist;
    out[2] = r.max_dist;
}

/* Object-level candidate generation exactly as the reference's filter runs it
 * (KNNJoin.cpp:553-573, WithinJoin.cpp:80-97, tile.cpp:76-85, tile_IO.cpp:47):
 * an octree over tile-2 object boxes (leaf size 10); for every tile-1 object a
 * best-first kNN (query_knn_fast) or a within query.  boxes are 6 floats
 * (low xyz, high xyz), transforms 3 floats.  self_join excludes the query
 * object itself, as the pointer test at octree.cpp:253/299 does.
 * Output: CSR offsets [n1+1] and ids in the reference's candidate order.
 * Returns the total number of candidates, or -1 if cap is too small. */
static long candidates_impl(const float *box1, const float *xf1, long n1,
                            const float *box2, const float *xf2, long n2,
                            int self_join, int knn, float within, int is_knn,
                            const int *qmap, long *off, int *ids, long cap)
{
    std::vector<weighted_aab> b2((size_t)n2);
    std::vector<weighted_aab *> ptr2((size_t)n2);
    tdbase::aab space;
    for (long i = 0; i < n2; ++i) {
        weighted_aab &w = b2[(size_t)i];
        w.set_box(box2[6 * i], box2[6 * i + 1], box2[6 * i + 2],
                  box2[6 * i + 3], box2[6 * i + 4], box2[6 * i + 5]);
        w.id = (int)i;
        w.transform[0] = xf2[3 * i];
        w.transform[1] = xf2[3 * i + 1];
        w.transform[2] = xf2[3 * i + 2];
        ptr2[(size_t)i] = &w;
        space.update(w);
    }
    OctreeNode *tree = new OctreeNode(space, 0, 10);
    for (long i = 0; i < n2; ++i) tree->addObject(ptr2[(size_t)i]);

    std::vector<weighted_aab> b1;
    if (!self_join) b1.resize((size_t)n1);
    long total = 0;
    off[0] = 0;
    for (long i = 0; i < n1; ++i) {
        weighted_aab *q;
        if (self_join) {
            q = ptr2[(size_t)(qmap ? qmap[i] : i)];
        } else {
            q = &b1[(size_t)i];
            q->set_box(box1[6 * i], box1[6 * i + 1], box1[6 * i + 2],
                       box1[6 * i + 3], box1[6 * i + 4], box1[6 * i + 5]);
            q->id = (int)i;
            q->transform[0] = xf1[3 * i];
            q->transform[1] = xf1[3 * i + 1];
            q->transform[2] = xf1[3 * i + 2];
        }
        std::vector<std::pair<int, range>> cand;
        float xf[3] = {xf1[3 * i], xf1[3 * i + 1], xf1[3 * i + 2]};
        if (is_knn == 2) {
            // intersect: SpatialJoin::mbb_intersect (IntersectionJoin.cpp:12-60)
            // sorts the octree's ids and skips duplicates
            std::vector<int> hit;
            tree->query_intersect(q, hit);
            std::sort(hit.begin(), hit.end());
            int former = -1;
            for (int id : hit) {
                if (id != former) cand.push_back({id, range()});
                former = id;
            }
        } else if (is_knn) {
            float mm = 3.4e38f;
            tree->query_knn_fast(q, xf, cand, mm, knn);
        } else {
            tree->query_within(q, xf, cand, within);
        }
        for (auto &c : cand) {
            if (total >= cap) { delete tree; return -1; }
            ids[total++] = c.first;
        }
        off[i + 1] = total;
    }
    delete tree;
    return total;
}

long tdr_candidates(const float *box1, const float *xf1, long n1,
                    const float *box2, const float *xf2, long n2,
                    int self_join, int knn, float within, int is_knn,
                    long *off, int *ids, long cap)
{
    return candidates_impl(box1, xf1, n1, box2, xf2, n2, self_join, knn, within, is_knn, nullptr, off, ids, cap);
}

/* The same for a chosen set of query objects: query i is tile-1 object
 * qmap[i] (its box and transform are box1[6 i..], xf1[3 i..]); in a self-join
 * the octree's pointer test excludes tile-2 object qmap[i]. */
long tdr_candidates_sel(const float *box1, const float *xf1, long n1,
                        const float *box2, const float *xf2, long n2,
                        int self_join, int knn, float within, int is_knn,
                        const int *qmap, long *off, int *ids, long cap)
{
    return candidates_impl(box1, xf1, n1, box2, xf2, n2, self_join, knn, within, is_knn, qmap, off, ids, cap);
}

} /* extern "C" */
