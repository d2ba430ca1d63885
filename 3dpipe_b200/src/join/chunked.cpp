// chunked.cpp -- a join whose tiles do not fit on the device (tdp_join_chunked).
//
// Both tiles stay in host memory as RAW bytes.  The object candidates are
// computed once on the host for the whole tiles (src/index: the same lists as
// the reference octree).  Tile 1 is then processed in contiguous chunks of
// query objects; for each chunk a RAW sub-tile of tile 2 is assembled from
// exactly the tile-2 objects that are candidates of the chunk, in increasing
// id, and both are attached (their triangles fetched by the join as it
// refines them), joined and freed.  Because the sub-tile holds
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
#include <atomic>
#include <cstdlib>
#include <thread>
#include <tuple>
#include <cstring>
#include <functional>
#include <future>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

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

// A host staging buffer, page-locked when possible (uploads then run at the
// full host-to-device rate), reused by every chunk assembled into it.
struct HostBuf {
    uint8_t* p = nullptr;
    size_t cap = 0;
    bool pinned = false;
    bool alloc(size_t bytes) {
        cap = bytes;
        pinned = cudaHostAlloc((void**)&p, bytes, cudaHostAllocDefault) == cudaSuccess;
        if (!pinned) p = (uint8_t*)std::malloc(bytes);
        return p != nullptr;
    }
    ~HostBuf() {
        if (!p) return;
        if (pinned) cudaFreeHost(p);
        else std::free(p);
    }
};

struct Chunk {
    long q0 = 0, q1 = 0;       // query objects [q0, q1)
    std::vector<int32_t> sub;  // global tile-2 ids in the sub-tile, increasing
    uint8_t* raw1 = nullptr;   // in the chunk's HostBuf: RAW chunk of tile 1, then the sub-tile
    uint8_t* raw2 = nullptr;
    size_t len1 = 0, len2 = 0;
};

// copy (dst, src, len) pieces with a few threads, split by bytes
void parallel_copy(std::vector<std::tuple<uint8_t*, const uint8_t*, size_t>>& pieces) {
    size_t total = 0;
    for (auto& x : pieces) total += std::get<2>(x);
    const unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (T == 1 || total < ((size_t)64 << 20)) {
        for (auto& x : pieces) std::memcpy(std::get<0>(x), std::get<1>(x), std::get<2>(x));
        return;
    }
    // cut big pieces so that every thread gets about total / T bytes
    std::vector<std::tuple<uint8_t*, const uint8_t*, size_t>> cut;
    const size_t part = total / T + 1;
    for (auto& x : pieces)
        for (size_t o = 0; o < std::get<2>(x); o += part)
            cut.emplace_back(std::get<0>(x) + o, std::get<1>(x) + o, std::min(part, std::get<2>(x) - o));
    std::vector<std::thread> th;
    std::atomic<size_t> next{0};
    for (unsigned t = 0; t < T; ++t)
        th.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < cut.size();)
                std::memcpy(std::get<0>(cut[i]), std::get<1>(cut[i]), std::get<2>(cut[i]));
        });
    for (auto& x : th) x.join();
}

void build_chunk(const uint8_t* b1, const TileHost& h1, const uint8_t* b2, const TileHost& h2,
                 const std::vector<int64_t>& off, const std::vector<int32_t>& ids, long q0, long q1, HostBuf& buf,
                 Chunk& c) {
    c.q0 = q0;
    c.q1 = q1;
    c.sub.assign(ids.begin() + off[q0], ids.begin() + off[q1]);
    std::sort(c.sub.begin(), c.sub.end());
    c.sub.erase(std::unique(c.sub.begin(), c.sub.end()), c.sub.end());
    const uint64_t s1 = rec_begin(h1, q0), e1 = rec_end(h1, q1 - 1);
    c.len1 = 1 + (e1 - s1);
    c.len2 = 1;
    for (int32_t o : c.sub) c.len2 += rec_end(h2, o) - rec_begin(h2, o);
    c.raw1 = buf.p;
    c.raw2 = buf.p + c.len1;
    c.raw1[0] = b1[0];
    c.raw2[0] = b2[0];
    std::vector<std::tuple<uint8_t*, const uint8_t*, size_t>> pieces;
    pieces.emplace_back(c.raw1 + 1, b1 + s1, e1 - s1);
    size_t p = 1;
    for (int32_t o : c.sub) {
        const uint64_t s = rec_begin(h2, o), n = rec_end(h2, o) - s;
        pieces.emplace_back(c.raw2 + p, b2 + s, n);
        p += n;
    }
    parallel_copy(pieces);
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
    if (prm->query_begin != 0 || prm->query_end >= 0)
        return fail(ctx, TDP_ERR_ARG, "a query range is not supported by the chunked join (it chunks the queries itself)");
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
    // chunk plan: grow each chunk object by object while the chunk, its
    // candidates' sub-tile and the join's scratch fit the context's budget
    // (about 2.5x their RAW bytes on the device: tiles, upload staging, join
    // state), at most chunk_objects per chunk
    std::vector<std::pair<long, long>> plan;
    double max_chunk_bytes = 0;
    {
        const double reserve = std::min(512.0 * (1 << 20), 0.25 * (double)ctx->budget);
        const double limit = ctx->budget ? ((double)ctx->budget - reserve) / 2.5 : 1e300;
        std::vector<char> mark((size_t)h2.n_obj, 0);
        std::vector<int32_t> touched;
        double bytes = 0;
        long q0 = 0;
        for (long q = 0; q < h1.n_obj; ++q) {
            double add = (double)(rec_end(h1, q) - rec_begin(h1, q));
            for (int64_t k = off[q]; k < off[q + 1]; ++k)
                if (!mark[ids[k]]) add += (double)(rec_end(h2, ids[k]) - rec_begin(h2, ids[k]));
            if (q > q0 && (q - q0 >= chunk_objects || bytes + add > limit)) {
                plan.push_back({q0, q});
                max_chunk_bytes = std::max(max_chunk_bytes, bytes);
                for (int32_t o : touched) mark[o] = 0;
                touched.clear();
                bytes = 0;
                q0 = q;
                add = (double)(rec_end(h1, q) - rec_begin(h1, q));
                for (int64_t k = off[q]; k < off[q + 1]; ++k)
                    if (!mark[ids[k]]) add += (double)(rec_end(h2, ids[k]) - rec_begin(h2, ids[k]));
            }
            for (int64_t k = off[q]; k < off[q + 1]; ++k)
                if (!mark[ids[k]]) { mark[ids[k]] = 1; touched.push_back(ids[k]); }
            bytes += add;
        }
        if (h1.n_obj > q0) plan.push_back({q0, h1.n_obj});
        max_chunk_bytes = std::max(max_chunk_bytes, bytes);
    }
    HostBuf bufs[2];
    for (HostBuf& b : bufs)
        if (!b.alloc((size_t)max_chunk_bytes + 64)) return fail(ctx, TDP_ERR_NOMEM, "cannot allocate host chunk buffers");
    auto make = [&](long q0, long q1, int slot) {
        auto c = std::make_unique<Chunk>();
        build_chunk(b1, h1, b2, h2, off, ids, q0, q1, bufs[slot], *c);
        return c;
    };
    // one chunk on the device; a chunk that exceeds the budget is split in two
    std::function<int(Chunk&, int)> run = [&](Chunk& c, int slot) -> int {
        ++inf.chunks;
        if (c.sub.empty()) return TDP_OK;  // no candidates: nothing to report
        tdp_tile *t1 = nullptr, *t2 = nullptr;
        tdp_result* r = nullptr;
        // a page-locked chunk buffer is attached: the join fetches only the
        // voxels it refines (and the buffer is not rewritten before the
        // chunk's tiles are freed); otherwise the chunk is uploaded whole
        auto load = [&](const uint8_t* raw, size_t len, tdp_tile** t) {
            return bufs[slot].pinned ? tdp_tile_attach(ctx, raw, len, 0, t) : tdp_tile_upload(ctx, raw, len, 0, t);
        };
        int rc = load(c.raw1, c.len1, &t1);
        if (rc == TDP_OK) rc = load(c.raw2, c.len2, &t2);
        if (rc == TDP_OK) rc = tdp_join(ctx, t1, t2, prm, &r);
        if (rc == TDP_OK) {
            tdp_tile_info i1{}, i2{};
            tdp_tile_get_info(t1, &i1);
            tdp_tile_get_info(t2, &i2);
            inf.h2d_bytes += (double)(i1.h2d_bytes + i2.h2d_bytes) + ctx->stats.fetch_bytes;
        }
        if (t1) tdp_tile_free(ctx, t1);
        if (t2) tdp_tile_free(ctx, t2);
        if (rc == TDP_ERR_NOMEM && c.q1 - c.q0 > 1) {
            --inf.chunks;
            ++inf.splits;
            // the halves reuse this chunk's buffer one after the other
            const long q0 = c.q0, mid = c.q0 + (c.q1 - c.q0) / 2, q1 = c.q1;
            auto lo = make(q0, mid, slot);
            if ((rc = run(*lo, slot)) != TDP_OK) return rc;
            auto hi = make(mid, q1, slot);
            return run(*hi, slot);
        }
        if (rc != TDP_OK) return rc;
        inf.tri_pairs += ctx->stats.tri_pairs;
        inf.join_ms += ctx->stats.total_ms;
        for (size_t i = 0; i < r->q.size(); ++i) {
            R->q.push_back(r->q[i] + (int)c.q0);
            R->t.push_back(c.sub[r->t[i]]);
            R->d.push_back(r->d[i]);
        }
        tdp_result_free(r);
        return TDP_OK;
    };
    std::future<std::unique_ptr<Chunk>> fut;
    if (!plan.empty()) fut = std::async(std::launch::async, make, plan[0].first, plan[0].second, 0);
    for (size_t k = 0; k < plan.size(); ++k) {
        std::unique_ptr<Chunk> c = fut.get();
        const int slot = (int)(k & 1);
        if (k + 1 < plan.size())  // the next chunk is assembled into the other buffer meanwhile
            fut = std::async(std::launch::async, make, plan[k + 1].first, plan[k + 1].second, 1 - slot);
        rc = run(*c, slot);
        if (rc != TDP_OK) {
            if (fut.valid()) fut.wait();
            return rc;
        }
    }
    size_t in_use = 0, peak = 0;
    tdp_ctx_memory(ctx, &in_use, &peak);
    inf.device_peak_bytes = (double)peak;
    if (info) *info = inf;
    *out = R.release();
    return TDP_OK;
}
