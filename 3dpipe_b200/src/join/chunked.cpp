// chunked.cpp -- a join whose tiles do not fit on the device (tdp_join_chunked).
//
// Both tiles stay in host memory as RAW bytes.  The object candidates are
// computed once on the host for the whole tiles (src/index: the same lists as
// the reference octree).  Tile 1 is then processed in contiguous chunks of
// query objects; for each chunk a RAW sub-tile of tile 2 is assembled from
// exactly the tile-2 objects that are candidates of the chunk, in increasing
// id, and both are uploaded, joined and freed.  Because the sub-tile holds
// every candidate of the chunk's queries and keeps their id order, each
// query's candidate list (set and order), and with it every filter decision,
// refine result and reported pair, is the one of the whole join; the result
// ids are mapped back to global ids.  A host thread assembles chunk k+1 while
// the device joins chunk k.
// The reference streams LOD data of a resident tile through pinned chunks
// (SpatialJoin::packing_data_stream, src/join/SpatialJoin.cpp:169-248) but
// needs both tiles decoded in host memory and its filter scratch on the
// device for the whole tile (src/geometry/computing_gpu.cu:4538-4626).
#include <algorithm>
#include <cstring>
#include <future>
#include <string>
#include <vector>

#include "../../csrc/ctx.cuh"
#include "index/candidates.h"
#include "join/result.h"
#include "storage/dev_tile.h"
#include "storage/dt_format.h"
#include "tdp.h"

namespace tdp {
namespace {

// byte range [begin, end) of object i's record
inline uint64_t rec_begin(const TileHost& h, long i) { return h.obj_data_off[i] - 8; }
inline uint64_t rec_end(const TileHost& h, long i) {
    const uint64_t nv = h.obj_vox_off[i + 1] - h.obj_vox_off[i];
    return h.obj_data_off[i] + h.obj_data_size[i] + 8 + kNumLods * 8 + nv * (9 * 4 + kNumLods * 16) + 12;
}

struct Chunk {
    long q0 = 0, q1 = 0;           // query objects [q0, q1)
    std::vector<int32_t> sub;       // global tile-2 ids in the sub-tile, increasing
    std::vector<uint8_t> raw1, raw2;
};

void build_chunk(const uint8_t* b1, const TileHost& h1, const uint8_t* b2, const TileHost& h2,
                 const std::vector<int64_t>& off, const std::vector<int32_t>& ids, long q0, long q1, Chunk& c) {
    c.q0 = q0;
    c.q1 = q1;
    c.sub.assign(ids.begin() + off[q0], ids.begin() + off[q1]);
    std::sort(c.sub.begin(), c.sub.end());
    c.sub.erase(std::unique(c.sub.begin(), c.sub.end()), c.sub.end());
    const uint64_t s1 = rec_begin(h1, q0), e1 = rec_end(h1, q1 - 1);
    c.raw1.resize(1 + (e1 - s1));
    c.raw1[0] = b1[0];
    std::memcpy(c.raw1.data() + 1, b1 + s1, e1 - s1);
    size_t bytes = 1;
    for (int32_t o : c.sub) bytes += rec_end(h2, o) - rec_begin(h2, o);
    c.raw2.resize(bytes);
    c.raw2[0] = b2[0];
    size_t p = 1;
    for (int32_t o : c.sub) {
        const uint64_t s = rec_begin(h2, o), n = rec_end(h2, o) - s;
        std::memcpy(c.raw2.data() + p, b2 + s, n);
        p += n;
    }
}

}  // namespace
}  // namespace tdp

using namespace tdp;

extern "C" int tdp_join_chunked(tdp_ctx* ctx, const void* raw1, size_t len1, const void* raw2, size_t len2,
                                const tdp_join_params* prm, long chunk_objects, tdp_chunked_info* info,
                                tdp_result** out) {
    if (!ctx || !raw1 || !raw2 || !prm || !out || chunk_objects < 1) return TDP_ERR_ARG;
    *out = nullptr;
    if (prm->obj_knn) return fail(ctx, TDP_ERR_ARG, "per-object queries are not supported by the chunked join");
    const uint8_t* b1 = (const uint8_t*)raw1;
    const uint8_t* b2 = (const uint8_t*)raw2;
    TileHost h1, h2;
    std::string err;
    int rc = parse_raw_dt(b1, len1, 0, h1, err);
    if (rc == TDP_OK) rc = parse_raw_dt(b2, len2, 0, h2, err);
    if (rc != TDP_OK) return fail(ctx, rc, err);
    const bool knn = prm->query == TDP_QUERY_NN, isect = prm->query == TDP_QUERY_INTERSECT;
    if (knn && prm->knn < 1) return fail(ctx, TDP_ERR_ARG, "knn must be >= 1");
    // global candidates, exactly as a whole join computes them
    CandidateQuery cq{h1.obj_box.data(), h1.obj_xf.data(), h1.n_obj, h2.obj_box.data(), h2.obj_xf.data(),
                      h2.n_obj, false, knn, knn ? prm->knn : 0, isect ? 0.f : prm->within_dist, 0};
    cq.strict_overlap = isect;
    std::vector<int64_t> off;
    std::vector<int32_t> ids;
    generate_candidates(cq, off, ids);
    tdp_chunked_info inf{};
    std::unique_ptr<tdp_result> R(new tdp_result());
    auto next_chunk = [&](long q0) {
        auto c = std::make_unique<Chunk>();
        build_chunk(b1, h1, b2, h2, off, ids, q0, std::min(h1.n_obj, q0 + chunk_objects), *c);
        return c;
    };
    std::future<std::unique_ptr<Chunk>> fut;
    if (h1.n_obj > 0) fut = std::async(std::launch::async, next_chunk, 0L);
    for (long q0 = 0; q0 < h1.n_obj; q0 += chunk_objects) {
        std::unique_ptr<Chunk> c = fut.get();
        const long q1n = q0 + chunk_objects;
        if (q1n < h1.n_obj) fut = std::async(std::launch::async, next_chunk, q1n);  // overlaps this chunk's join
        ++inf.chunks;
        inf.h2d_bytes += (double)(c->raw1.size() + c->raw2.size());
        if (c->sub.empty()) continue;  // no candidates: nothing to report
        tdp_tile *t1 = nullptr, *t2 = nullptr;
        tdp_result* r = nullptr;
        rc = tdp_tile_upload(ctx, c->raw1.data(), c->raw1.size(), 0, &t1);
        if (rc == TDP_OK) rc = tdp_tile_upload(ctx, c->raw2.data(), c->raw2.size(), 0, &t2);
        if (rc == TDP_OK) rc = tdp_join(ctx, t1, t2, prm, &r);
        if (t1) tdp_tile_free(ctx, t1);
        if (t2) tdp_tile_free(ctx, t2);
        if (rc != TDP_OK) {
            if (fut.valid()) fut.wait();
            return rc;
        }
        inf.tri_pairs += ctx->stats.tri_pairs;
        inf.join_ms += ctx->stats.total_ms;
        for (size_t i = 0; i < r->q.size(); ++i) {
            R->q.push_back(r->q[i] + (int)c->q0);
            R->t.push_back(c->sub[r->t[i]]);
            R->d.push_back(r->d[i]);
        }
        tdp_result_free(r);
    }
    size_t in_use = 0, peak = 0;
    tdp_ctx_memory(ctx, &in_use, &peak);
    inf.device_peak_bytes = (double)peak;
    if (info) *info = inf;
    *out = R.release();
    return TDP_OK;
}
