// server.cpp -- continuous-batching request loop over a resident tile 2
// (tdp_server_* in include/tdp.h).
//
// Two device arenas hold the query objects of the admitted requests.  An
// arena is a tdp_tile whose device arrays are allocated once at full
// capacity.  A request's RAW bytes, and its metadata in request-local
// offsets (voxel records, CSR offsets, Hausdorff values, unpack segments,
// built on the host into a page-locked block), are first copied to one of
// two device staging areas that belong to no arena (the slow PCIe part; the
// next request's copy runs while the current one is appended).  Appending is
// then device work only, on the arena's stream: a commit kernel writes the
// metadata at the arena's running offsets (objects, voxels, triangles per
// LOD) and the tile-upload kernel unpacks the triangles from the staging area.
// No host-to-device copy happens while an arena is being appended to, so an
// append never queues behind a staging copy on the copy engine.
//
//   admitter thread   takes requests in arrival order, stages each one, then
//                     appends it to the arena being filled if it fits
//                     (admission by memory); a request that does not fit
//                     seals the arena and waits for the other one;
//   executor thread   whenever it is idle, takes the sealed arena or else the
//                     filling one (if it holds a request), waits on the
//                     arena's upload event, runs ONE tdp_join over all of its
//                     objects with per-object queries (obj_knn / obj_within),
//                     splits the rows by request and frees the arena.
// While a batch runs, arrivals go into the other arena, so uploads overlap
// the join and the next batch starts as soon as the GPU is free.
// The reference has no request loop (one join per `tdbase join` run,
// src/tools/tdbase.cpp:482-549).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../csrc/ctx.cuh"
#include "../../csrc/serve_kernels.cuh"
#include "../../csrc/tile_kernels.cuh"
#include "join/result.h"
#include "storage/dev_tile.h"
#include "storage/dt_format.h"
#include "tdp.h"

namespace tdp {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    uint64_t id = 0;
    const uint8_t* raw = nullptr;
    size_t len = 0;
    TileHost host;     // parsed at submit
    uint64_t base = 0; // byte offset of the first object's record in raw
    uint64_t span = 0; // bytes from base to the end of the last object's data
    const uint8_t* dev = nullptr;  // device view of raw when it is page-locked
    bool fetched = false;          // the join fetches its triangles from raw (else staged whole)
    double staged_bytes = 0;       // bytes its staging copies moved
    int knn = 0;       // > 0: kNN; 0: within
    float within = 0.f;
    Clock::time_point t_submit, t_start, t_done;
    long o0 = 0;       // first object in its arena
    long batch = -1;
    int batch_requests = 0;
    int status = TDP_OK;
    bool done = false;
    std::unique_ptr<tdp_result> res;
};

enum class ArenaState { kFree, kFilling, kSealed, kRunning };

struct Arena {
    tdp_tile tile;                 // device arrays at capacity; counts grow with appends
    uint32_t n_tri[kNumLods] = {};
    std::vector<Request*> reqs;
    ArenaState state = ArenaState::kFree;
    bool appending = false;
    cudaStream_t up = nullptr;
    cudaEvent_t ready = nullptr;
};

// Byte layout of one request's staged metadata (every section 16-byte aligned).
struct MetaLayout {
    size_t vox = 0, obj_vox = 0, obj_hd = 0, obj_phd = 0, vtri[kNumLods] = {}, data_abs = 0, segs = 0, bytes = 0;
    long nseg = 0;
};

size_t up16(size_t x) { return (x + 15) & ~(size_t)15; }

MetaLayout meta_layout(long n, long nv, long nseg) {
    MetaLayout L;
    size_t o = 0;
    L.vox = o; o = up16(o + (size_t)nv * 3 * sizeof(float4));
    L.obj_vox = o; o = up16(o + (size_t)(n + 1) * 4);
    L.obj_hd = o; o = up16(o + (size_t)n * kNumLods * 4);
    L.obj_phd = o; o = up16(o + (size_t)n * kNumLods * 4);
    for (int l = 0; l < kNumLods; ++l) { L.vtri[l] = o; o = up16(o + (size_t)(nv + 1) * 4); }
    L.data_abs = o; o = up16(o + (size_t)n * 8);
    L.segs = o; o = up16(o + (size_t)nseg * sizeof(UnpackSeg));
    L.bytes = o;
    L.nseg = nseg;
    return L;
}

}  // namespace
}  // namespace tdp

using namespace tdp;

struct tdp_server {
    tdp_ctx* ctx = nullptr;
    const tdp_tile* t2 = nullptr;
    tdp_server_params p{};
    Arena arena[2];
    uint8_t* stage[2] = {};           // device staging of RAW bytes (double-buffered)
    uint8_t* dmeta[2] = {};           // device staging of the metadata
    uint8_t* hmeta[2] = {};           // page-locked host metadata blocks
    size_t meta_cap = 0;
    MetaLayout meta[2];
    cudaEvent_t staged[2] = {};       // a stage's copies finished
    cudaStream_t copy = nullptr;      // stream of the staging copies
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> table;
    uint64_t next_id = 1;
    long batches = 0, completed = 0, failed = 0, split_batches = 0;
    double busy_ms = 0, upload_ms = 0, upload_bytes = 0, fetch_bytes = 0;
    bool stop = false;
    std::thread admitter, executor;
};

namespace {

void reset_arena(Arena& a) {
    TileHost& H = a.tile.host;
    a.tile.boxes_n = 0;
    a.tile.n_obj = a.tile.n_vox = 0;
    H.n_obj = H.n_vox = 0;
    H.obj_box.clear();
    H.obj_xf.clear();
    for (int l = 0; l < kNumLods; ++l) {
        a.n_tri[l] = 0;
        H.n_tris[l] = 0;
    }
    a.reqs.clear();
}

bool fits(const tdp_server* S, const Arena& a, const Request& r) {
    if (a.tile.n_obj + r.host.n_obj > S->p.arena_objects) return false;
    if (a.tile.n_vox + r.host.n_vox > S->p.arena_voxels) return false;
    for (int l = 0; l < kNumLods; ++l)
        if ((long)a.n_tri[l] + (long)r.host.n_tris[l] > S->p.arena_tris) return false;
    return true;
}

// Build r's metadata (request-local offsets) into hmeta[j] and start copying
// it and r's RAW bytes into staging area j (copy stream, asynchronous).
// Returns TDP_OK or an error for malformed triangle blocks.
int start_copy(tdp_server* S, Request* r, int j) {
    const TileHost& h = r->host;
    const long n = h.n_obj, nv = h.n_vox;
    long nseg = 0;
    if (!r->fetched)
        for (int l = 0; l < kNumLods; ++l)
            for (long v = 0; v < nv; ++v) nseg += h.vox_cnt[l][v] != 0;
    const MetaLayout L = meta_layout(n, nv, nseg);
    if (L.bytes > S->meta_cap) return TDP_ERR_ARG;
    uint8_t* m = S->hmeta[j];
    float4* vox = (float4*)(m + L.vox);
    for (long v = 0; v < nv; ++v) {
        const float* b = &h.vox_box[9 * v];
        vox[3 * v + 0] = make_float4(b[0], b[1], b[2], 0.f);
        vox[3 * v + 1] = make_float4(b[3], b[4], b[5], 0.f);
        vox[3 * v + 2] = make_float4(b[6], b[7], b[8], 0.f);
    }
    std::memcpy(m + L.obj_vox, h.obj_vox_off.data(), (size_t)(n + 1) * 4);
    std::memcpy(m + L.obj_hd, h.obj_hd.data(), (size_t)n * kNumLods * 4);
    std::memcpy(m + L.obj_phd, h.obj_phd.data(), (size_t)n * kNumLods * 4);
    uint64_t* abs = (uint64_t*)(m + L.data_abs);
    for (long o = 0; o < n; ++o) abs[o] = r->fetched ? (uint64_t)(uintptr_t)(r->dev + h.obj_data_off[o]) : 0;
    UnpackSeg* seg = (UnpackSeg*)(m + L.segs);
    long k = 0;
    for (int l = 0; l < kNumLods; ++l) {
        uint32_t* vt = (uint32_t*)(m + L.vtri[l]);
        vt[0] = 0;
        for (long v = 0; v < nv; ++v) {
            const uint32_t c = h.vox_cnt[l][v];
            vt[v + 1] = vt[v] + c;
            if (!c || r->fetched) continue;
            const uint64_t src = h.vox_byte_off[l][v] - r->base;
            if ((src & 3u) || src + (uint64_t)c * 44 > r->span) return TDP_ERR_FORMAT;
            seg[k++] = UnpackSeg{src, vt[v], c | ((uint32_t)l << 24)};  // dst local to the request
        }
    }
    S->meta[j] = L;
    // a page-locked request moves only its metadata now; its triangles are
    // fetched by the join, voxel by voxel, from the caller's buffer
    r->staged_bytes = (double)L.bytes + (r->fetched ? 0.0 : (double)r->span);
    if (cudaMemcpyAsync(S->dmeta[j], m, L.bytes, cudaMemcpyHostToDevice, S->copy) != cudaSuccess ||
        (!r->fetched &&
         cudaMemcpyAsync(S->stage[j], r->raw + r->base, r->span, cudaMemcpyHostToDevice, S->copy) != cudaSuccess) ||
        cudaEventRecord(S->staged[j], S->copy) != cudaSuccess)
        return TDP_ERR_CUDA;
    return TDP_OK;
}

// Append the request staged in area j at the arena's offsets: device work on
// the arena's stream only (admitter thread; the arena is not visible to the
// executor while `appending` is set).
int append(tdp_server* S, Arena& a, Request& r, int j) {
    const TileHost& h = r.host;
    TileHost& H = a.tile.host;
    const long o0 = a.tile.n_obj, v0 = a.tile.n_vox, n = h.n_obj, nv = h.n_vox;
    uint32_t t0[kNumLods];
    for (int l = 0; l < kNumLods; ++l) t0[l] = a.n_tri[l];
    const MetaLayout& L = S->meta[j];
    const uint8_t* m = S->dmeta[j];
    ArenaMeta am{(const float4*)(m + L.vox), (const uint32_t*)(m + L.obj_vox), (const float*)(m + L.obj_hd),
                 (const float*)(m + L.obj_phd), {}, (const uint64_t*)(m + L.data_abs), r.fetched ? 1u : 0u};
    ArenaDst ad{a.tile.vox, a.tile.obj_vox, a.tile.obj_hd, a.tile.obj_phd, {},
                a.tile.lazy_data_off, a.tile.lazy_state, a.tile.lazy_stride};
    float4* tri_at[kNumLods];
    for (int l = 0; l < kNumLods; ++l) {
        am.vtri[l] = (const uint32_t*)(m + L.vtri[l]);
        ad.vtri[l] = a.tile.vtri[l];
        tri_at[l] = a.tile.tri[l] + 3 * (size_t)t0[l];  // segments carry request-local destinations
    }
    cudaError_t e = launch_arena_commit(am, ad, n, nv, o0, v0, t0, S->ctx->num_sms, a.up);
    if (e == cudaSuccess && L.nseg > 0)
        e = launch_unpack(S->stage[j], (const UnpackSeg*)(m + L.segs), (int)L.nseg, tri_at, S->ctx->num_sms, a.up);
    if (e == cudaSuccess) e = cudaEventRecord(a.ready, a.up);
    // the staging area is refilled two requests later: finish with it now
    if (e == cudaSuccess) e = cudaStreamSynchronize(a.up);
    if (e != cudaSuccess) return TDP_ERR_CUDA;
    // host side of the arena: what the join reads from the host
    H.obj_box.insert(H.obj_box.end(), h.obj_box.begin(), h.obj_box.end());
    H.obj_xf.insert(H.obj_xf.end(), h.obj_xf.begin(), h.obj_xf.end());
    for (int l = 0; l < kNumLods; ++l) {
        a.n_tri[l] = t0[l] + (uint32_t)h.n_tris[l];
        H.n_tris[l] = a.n_tri[l];
    }
    a.tile.n_obj = H.n_obj = o0 + n;
    a.tile.n_vox = H.n_vox = v0 + nv;
    a.tile.boxes_n = 0;  // the device copy of the boxes is stale
    return TDP_OK;
}

// A request can be fetched from by the join when its bytes are page-locked
// from the first to the last and every object keeps its voxels' triangles LOD
// by LOD and voxel by voxel (the writer's layout, src/storage/tile_IO.cpp:79-172).
bool fetchable(const uint8_t* raw, size_t len, const TileHost& h, const uint8_t** dev) {
    cudaPointerAttributes a0{}, a1{};
    void* dp = nullptr;
    if (len == 0 || cudaPointerGetAttributes(&a0, raw) != cudaSuccess || a0.type != cudaMemoryTypeHost ||
        cudaPointerGetAttributes(&a1, raw + len - 1) != cudaSuccess || a1.type != cudaMemoryTypeHost ||
        cudaHostGetDevicePointer(&dp, (void*)raw, 0) != cudaSuccess || !dp) {
        cudaGetLastError();
        return false;
    }
    if (h.first_noncanonical >= 0) return false;  // checked by the parser
    *dev = (const uint8_t*)dp;
    return true;
}

// Estimated join time of a request on its own, from the serving workload's
// per-nucleus costs on a B200 (5,000-nucleus requests against 1,000 vessels:
// kNN 0.25 + 0.107 K us per nucleus for K = 1..50, within about 0.5 us).
// Only the split of a batch into a small and a big pass reads it.
double estimated_ms(const Request& r) {
    const double per = r.knn > 0 ? 0.25 + 0.107 * r.knn : 0.5;
    return 1e-3 * per * (double)r.host.n_obj;
}

void finish(tdp_server* S, Request* r, int status) {
    r->status = status;
    r->t_done = Clock::now();
    r->done = true;
    ++S->completed;
    if (status != TDP_OK) ++S->failed;
}

void admitter_loop(tdp_server* S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    Request* cur = nullptr;  // request whose bytes are in (or on their way to) staging area j
    int j = 0;
    Clock::time_point t_cur;
    int cur_rc = TDP_OK;
    for (;;) {
        if (!cur) {
            S->cv.wait(lk, [&] { return S->stop || !S->pending.empty(); });
            if (S->stop) return;
            cur = S->pending.front();
            S->pending.pop_front();
            t_cur = Clock::now();
            lk.unlock();
            cur_rc = start_copy(S, cur, j);
            lk.lock();
        }
        // 1. the next request's bytes go to the other stage while this one is appended
        Request* nxt = nullptr;
        int nxt_rc = TDP_OK;
        Clock::time_point t_nxt;
        if (!S->pending.empty()) {
            nxt = S->pending.front();
            S->pending.pop_front();
        }
        lk.unlock();
        if (nxt) {
            t_nxt = Clock::now();
            nxt_rc = start_copy(S, nxt, 1 - j);
        }
        if (cur_rc == TDP_OK && cudaEventSynchronize(S->staged[j]) != cudaSuccess) cur_rc = TDP_ERR_CUDA;
        lk.lock();
        Request* r = cur;
        if (cur_rc != TDP_OK) {
            finish(S, r, cur_rc);
            S->cv.notify_all();
        } else {
            // 2. an arena with room: the one being filled, else a free one
            Arena* a = nullptr;
            for (;;) {
                S->cv.wait(lk, [&] {
                    if (S->stop) return true;
                    for (Arena& x : S->arena)
                        if (x.state == ArenaState::kFilling) { a = &x; return true; }
                    for (Arena& x : S->arena)
                        if (x.state == ArenaState::kFree) { a = &x; return true; }
                    return false;
                });
                if (S->stop) break;
                if (a->state == ArenaState::kFree) a->state = ArenaState::kFilling;
                if (fits(S, *a, *r)) break;
                a->state = ArenaState::kSealed;  // the executor takes it next
                a = nullptr;
                S->cv.notify_all();
            }
            if (!a) {
                finish(S, r, TDP_ERR_STATE);
                if (nxt) {
                    lk.unlock();
                    cudaEventSynchronize(S->staged[1 - j]);  // its copy may still read the caller's bytes
                    lk.lock();
                    finish(S, nxt, TDP_ERR_STATE);
                }
                S->cv.notify_all();
                return;
            }
            // 3. metadata and unpack into the arena (short)
            a->appending = true;
            r->o0 = a->tile.n_obj;
            lk.unlock();
            const int rc = append(S, *a, *r, j);
            const double up_ms = ms_between(t_cur, Clock::now());
            lk.lock();
            S->upload_ms += up_ms;
            S->upload_bytes += r->staged_bytes;
            a->appending = false;
            if (rc == TDP_OK) a->reqs.push_back(r);
            else finish(S, r, rc);
            S->cv.notify_all();
        }
        cur = nxt;
        cur_rc = nxt_rc;
        t_cur = t_nxt;
        j = 1 - j;
    }
}

void executor_loop(tdp_server* S) {
    tdp_ctx* ctx = S->ctx;
    cudaSetDevice(ctx->device);
    std::vector<int> obj_knn;
    std::vector<float> obj_within;
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        Arena* a = nullptr;
        S->cv.wait(lk, [&] {
            for (Arena& x : S->arena)
                if (x.state == ArenaState::kSealed && !x.appending) { a = &x; return true; }
            for (Arena& x : S->arena)
                if (x.state == ArenaState::kFilling && !x.appending && !x.reqs.empty()) { a = &x; return true; }
            return S->stop;
        });
        if (!a) return;  // stopping with nothing admitted left to run
        a->state = ArenaState::kRunning;
        const long batch = S->batches++;
        const auto t_start = Clock::now();
        for (Request* r : a->reqs) {
            r->t_start = t_start;
            r->batch = batch;
            r->batch_requests = (int)a->reqs.size();
        }
        std::vector<Request*> reqs = a->reqs;
        lk.unlock();
        // Small requests first: when a batch mixes requests whose estimated
        // join time exceeds big_request_ms with smaller ones, it runs as two joins over
        // the arena -- the small requests' objects with their queries and the
        // big ones' as within-0 (nearly free), then the reverse -- and each
        // request completes with its own pass.  A query object's result does
        // not depend on the other objects' queries, so the rows are the ones
        // a single join gives.
        std::vector<Request*> small, big;
        const double big_ms = S->p.big_request_ms;
        for (Request* r : reqs) (big_ms > 0.0 && estimated_ms(*r) > big_ms ? big : small).push_back(r);
        std::vector<std::vector<Request*>> passes;
        if (!small.empty() && !big.empty()) passes = {small, big};
        else passes = {reqs};
        if (passes.size() > 1) {
            lk.lock();
            ++S->split_batches;
            lk.unlock();
        }
        const long n = a->tile.n_obj;
        int rc = cudaStreamWaitEvent(ctx->stream, a->ready, 0) == cudaSuccess ? TDP_OK : TDP_ERR_CUDA;
        double fetched = 0.0;
        size_t done_passes = 0;  // passes whose requests are finished (a finished request may be freed at once)
        for (const std::vector<Request*>& pass : passes) {
            if (rc != TDP_OK) break;
            // per-object queries of this pass
            obj_knn.assign(n, 0);
            obj_within.assign(n, 0.f);
            for (Request* r : pass)
                for (long i = 0; i < r->host.n_obj; ++i) {
                    obj_knn[r->o0 + i] = r->knn;
                    obj_within[r->o0 + i] = r->within;
                }
            tdp_join_params jp;
            tdp_join_default_params(&jp);
            std::memcpy(jp.lods, S->p.lods, sizeof(jp.lods));
            jp.n_lods = S->p.n_lods;
            jp.hausdorff_level = S->p.hausdorff_level;
            jp.form = S->p.form;
            jp.obj_knn = obj_knn.data();
            jp.obj_within = obj_within.data();
            tdp_result* res = nullptr;
            if (rc == TDP_OK) rc = tdp_join(ctx, &a->tile, S->t2, &jp, &res);
            if (rc == TDP_OK) fetched += ctx->stats.fetch_bytes;
            // split the rows (sorted by query object) by request
            if (rc == TDP_OK) {
                for (Request* r : pass) {
                    r->res.reset(new tdp_result());
                    const long lo = r->o0, hi = r->o0 + r->host.n_obj;
                    auto b = std::lower_bound(res->q.begin(), res->q.end(), (int)lo);
                    auto e = std::lower_bound(res->q.begin(), res->q.end(), (int)hi);
                    const size_t i0 = b - res->q.begin(), i1 = e - res->q.begin();
                    r->res->q.reserve(i1 - i0);
                    for (size_t i = i0; i < i1; ++i) r->res->q.push_back(res->q[i] - (int)lo);
                    r->res->t.assign(res->t.begin() + i0, res->t.begin() + i1);
                    r->res->d.assign(res->d.begin() + i0, res->d.begin() + i1);
                }
            }
            delete res;
            if (&pass != &passes.back() && rc == TDP_OK) {  // this pass's requests are done
                lk.lock();
                for (Request* r : pass) finish(S, r, rc);
                S->cv.notify_all();
                lk.unlock();
                ++done_passes;
            }
        }
        const double busy = ms_between(t_start, Clock::now());
        lk.lock();
        S->busy_ms += busy;
        S->fetch_bytes += fetched;
        for (size_t k = done_passes; k < passes.size(); ++k)
            for (Request* r : passes[k]) finish(S, r, rc);
        reset_arena(*a);
        a->state = ArenaState::kFree;
        S->cv.notify_all();
    }
}

}  // namespace

extern "C" {

void tdp_server_default_params(tdp_server_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->arena_objects = 65536;
    p->arena_voxels = 1L << 20;
    p->arena_tris = 1L << 25;
    p->max_request_bytes = (size_t)1 << 30;
    p->hausdorff_level = 2;
    p->form = TDP_FORM_TUNED;
    p->big_request_ms = 4.0;
}

int tdp_server_create(tdp_ctx* ctx, const tdp_tile* t2, const tdp_server_params* p, tdp_server** out) {
    if (!ctx || !t2 || !p || !out) return TDP_ERR_ARG;
    *out = nullptr;
    if (p->arena_objects < 1 || p->arena_voxels < 1 || p->arena_tris < 1 || p->arena_tris >= (1L << 32) ||
        p->max_request_bytes < 16)
        return fail(ctx, TDP_ERR_ARG, "server capacities must be positive (arena_tris < 2^32)");
    cudaSetDevice(ctx->device);
    std::unique_ptr<tdp_server> S(new tdp_server());
    S->ctx = ctx;
    S->t2 = t2;
    S->p = *p;
    S->meta_cap = meta_layout(p->arena_objects, p->arena_voxels, p->arena_voxels * kNumLods).bytes;
    for (Arena& a : S->arena) {
        tdp_tile& T = a.tile;
        T.device = ctx->device;
        auto alloc = [&](void** ptr, size_t bytes) {
            if (dmalloc(ctx, ptr, bytes) != cudaSuccess) return false;
            T.device_bytes += bytes;
            return true;
        };
        bool ok = alloc((void**)&T.vox, (size_t)p->arena_voxels * 3 * sizeof(float4)) &&
                  alloc((void**)&T.obj_vox, (size_t)(p->arena_objects + 1) * 4) &&
                  alloc((void**)&T.obj_hd, (size_t)p->arena_objects * kNumLods * 4) &&
                  alloc((void**)&T.obj_phd, (size_t)p->arena_objects * kNumLods * 4);
        for (int l = 0; ok && l < kNumLods; ++l)
            ok = alloc((void**)&T.tri[l], (size_t)p->arena_tris * 3 * sizeof(float4)) &&
                 alloc((void**)&T.vtri[l], (size_t)(p->arena_voxels + 1) * 4);
        // fetch state of the arena: requests in page-locked memory are fetched
        // by the join, the others are unpacked from staging (state 1)
        ok = ok && alloc((void**)&T.lazy_data_off, (size_t)p->arena_objects * 8) &&
             alloc((void**)&T.lazy_state, (size_t)kNumLods * p->arena_voxels * sizeof(unsigned)) &&
             alloc((void**)&T.lazy_bytes, sizeof(unsigned long long));
        T.lazy_on = true;
        T.lazy_raw = nullptr;  // lazy_data_off holds absolute addresses
        T.lazy_stride = p->arena_voxels;
        if (!ok || cudaStreamCreateWithFlags(&a.up, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&a.ready, cudaEventDisableTiming) != cudaSuccess) {
            tdp_server_destroy(S.release());
            return fail(ctx, TDP_ERR_NOMEM, "cannot allocate the serving arenas");
        }
        // the first entry of each CSR array stays 0
        cudaMemsetAsync(T.obj_vox, 0, 4, a.up);
        for (int l = 0; l < kNumLods; ++l) cudaMemsetAsync(T.vtri[l], 0, 4, a.up);
        cudaEventRecord(a.ready, a.up);
        TileHost& H = T.host;
        H.obj_box.reserve((size_t)p->arena_objects * 6);
        H.obj_xf.reserve((size_t)p->arena_objects * 3);
        reset_arena(a);
        if (cudaStreamSynchronize(a.up) != cudaSuccess) {
            tdp_server_destroy(S.release());
            return fail(ctx, TDP_ERR_CUDA, "serving arena set-up failed");
        }
    }
    if (dmalloc(ctx, (void**)&S->stage[0], p->max_request_bytes + 16) != cudaSuccess ||
        dmalloc(ctx, (void**)&S->stage[1], p->max_request_bytes + 16) != cudaSuccess ||
        dmalloc(ctx, (void**)&S->dmeta[0], S->meta_cap) != cudaSuccess ||
        dmalloc(ctx, (void**)&S->dmeta[1], S->meta_cap) != cudaSuccess ||
        cudaHostAlloc((void**)&S->hmeta[0], S->meta_cap, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&S->hmeta[1], S->meta_cap, cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->staged[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->staged[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking) != cudaSuccess) {
        tdp_server_destroy(S.release());
        return fail(ctx, TDP_ERR_NOMEM, "cannot allocate the serving staging buffer");
    }
    tdp_server* raw = S.release();
    raw->admitter = std::thread(admitter_loop, raw);
    raw->executor = std::thread(executor_loop, raw);
    *out = raw;
    return TDP_OK;
}

int tdp_server_submit(tdp_server* S, const void* raw_dt, size_t len, int query, int knn, float within,
                      uint64_t* id) {
    if (!S || !raw_dt || !id) return TDP_ERR_ARG;
    if (query == TDP_QUERY_NN ? knn < 1 : (query != TDP_QUERY_WITHIN || !(within >= 0.f))) return TDP_ERR_ARG;
    std::unique_ptr<Request> r(new Request());
    r->t_submit = Clock::now();
    r->raw = (const uint8_t*)raw_dt;
    r->len = len;
    std::string err;
    int rc = parse_raw_dt(r->raw, len, 0, r->host, err);
    if (rc != TDP_OK) return rc;
    const TileHost& h = r->host;
    if (h.n_obj < 1) return TDP_ERR_FORMAT;
    r->base = h.obj_data_off[0] - 8;  // the first object's first byte
    r->span = h.obj_data_off[h.n_obj - 1] + h.obj_data_size[h.n_obj - 1] - r->base;
    if (h.n_obj > S->p.arena_objects || h.n_vox > S->p.arena_voxels || r->span > S->p.max_request_bytes)
        return TDP_ERR_ARG;
    for (int l = 0; l < kNumLods; ++l)
        if ((long)h.n_tris[l] > S->p.arena_tris) return TDP_ERR_ARG;
    r->knn = query == TDP_QUERY_NN ? knn : 0;
    r->within = query == TDP_QUERY_NN ? 0.f : within;
    r->fetched = fetchable(r->raw, len, h, &r->dev);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return TDP_ERR_STATE;
    r->id = S->next_id++;
    *id = r->id;
    S->pending.push_back(r.get());
    S->table.emplace(r->id, std::move(r));
    S->cv.notify_all();
    return TDP_OK;
}

int tdp_server_wait(tdp_server* S, uint64_t id, int timeout_ms, tdp_result** result, tdp_request_info* info) {
    if (!S) return TDP_ERR_ARG;
    if (result) *result = nullptr;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->table.find(id);
    if (it == S->table.end()) return TDP_ERR_ARG;
    Request* r = it->second.get();
    auto done = [&] { return r->done; };
    if (timeout_ms < 0) S->cv.wait(lk, done);
    else if (!S->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return TDP_ERR_TIMEOUT;
    if (info) {
        info->queue_ms = r->batch >= 0 ? ms_between(r->t_submit, r->t_start) : 0.0;
        info->latency_ms = ms_between(r->t_submit, r->t_done);
        info->batch = r->batch;
        info->batch_requests = r->batch_requests;
        info->status = r->status;
    }
    const int status = r->status;
    if (status == TDP_OK && result) *result = r->res.release();
    S->table.erase(it);
    return status;
}

int tdp_server_get_stats(const tdp_server* S, tdp_server_stats* o) {
    if (!S || !o) return TDP_ERR_ARG;
    std::lock_guard<std::mutex> lk(const_cast<tdp_server*>(S)->mu);
    o->batches = S->batches;
    o->split_batches = S->split_batches;
    o->requests = S->completed;
    o->failed = S->failed;
    o->busy_ms = S->busy_ms;
    o->upload_ms = S->upload_ms;
    o->upload_bytes = S->upload_bytes;
    o->fetch_bytes = S->fetch_bytes;
    return TDP_OK;
}

int tdp_server_destroy(tdp_server* S) {
    if (!S) return TDP_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->admitter.joinable()) S->admitter.join();
    if (S->executor.joinable()) S->executor.join();
    tdp_ctx* ctx = S->ctx;
    cudaSetDevice(ctx->device);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (Request* r : S->pending)
            if (!r->done) finish(S, r, TDP_ERR_STATE);
        for (Arena& a : S->arena)
            for (Request* r : a.reqs)
                if (!r->done) finish(S, r, TDP_ERR_STATE);
        S->cv.notify_all();
    }
    for (Arena& a : S->arena) {
        if (a.up) cudaStreamSynchronize(a.up);
        tdp_tile& T = a.tile;
        dfree(ctx, T.vox); dfree(ctx, T.obj_vox); dfree(ctx, T.obj_hd); dfree(ctx, T.obj_phd);
        dfree(ctx, T.d_boxes);
        dfree(ctx, (void*)T.lazy_data_off); dfree(ctx, T.lazy_state); dfree(ctx, T.lazy_bytes);
        for (int l = 0; l < kNumLods; ++l) { dfree(ctx, T.tri[l]); dfree(ctx, T.vtri[l]); }
        if (a.ready) cudaEventDestroy(a.ready);
        if (a.up) cudaStreamDestroy(a.up);
    }
    if (S->copy) cudaStreamSynchronize(S->copy);
    for (int k = 0; k < 2; ++k) {
        dfree(ctx, S->stage[k]);
        dfree(ctx, S->dmeta[k]);
        if (S->hmeta[k]) cudaFreeHost(S->hmeta[k]);
        if (S->staged[k]) cudaEventDestroy(S->staged[k]);
    }
    if (S->copy) cudaStreamDestroy(S->copy);
    delete S;
    return TDP_OK;
}

}  // extern "C"
