// join_driver.cpp -- host orchestration of the spatial join (tdp_join).
//
// Follows the reference's chunked joins step for step, with all state in HBM:
//   SpatialJoin::nearest_neighbor_chunking   src/join/KNNJoin.cpp:1524-1811
//   SpatialJoin::within_chunking             src/join/WithinJoin.cpp:644-813
//   mbb_knn_op_gpu_one_kernel / mbb_within_op_gpu_one_kernel (the filter)
//                                            KNNJoin.cpp:497-851, WithinJoin.cpp:26-258
// 1. object candidates (GPU grid search, or the host grid in src/index), a CSR of object pairs;
// 2. filter: object ranges from all voxel pairs, kNN rank rule or within
//    classification, compaction of the voxel pairs that can still matter;
// 3. per LOD: refine every live, non-empty voxel pair, update voxel and
//    object ranges (with eviction), decide; stop when nothing is undecided.
// The host only reads a few counters per LOD; no triangle ever crosses PCIe.
//
// Forms: TDP_FORM_PLAIN uses the reference's FP32 decision rules and the
// one-CTA-per-voxel-pair refine; TDP_FORM_TUNED uses the persistent culled
// refine and decides only outside each range's FP32 error band.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../csrc/ctx.cuh"
#include "../../csrc/join_kernels.cuh"
#include "../../csrc/cand_kernels.cuh"
#include "../../csrc/exact_kernels.cuh"
#include "../../csrc/fetch_kernels.cuh"
#include "../../csrc/refine.cuh"
#include "index/candidates.h"
#include "storage/dev_tile.h"
#include "tdp.h"

#include "join/result.h"

namespace tdp {

namespace {

enum Slot {
    kPq = 20, kPt, kQoff, kPmn, kPmx, kPerr, kPstat, kPvp, kQconf, kCnt, kScanTmp, kRankSt,
    kVpa, kVpb, kVpair, kVmn, kVmx, kVerr, kValive, kVupd, kItems, kItemVp, kRes, kOutQ, kOutT, kOutD,
    kVexact, kPexact, kRes64,
    kKeyA = 60, kKeyB, kValA, kValB,  // result sort (50-59 hold the candidate buffers)
    kPexOut = 76, kOutD64,            // exact distances (64-75 and 78-81 are the exact stage's own)
    kQk = 82, kQtau,                  // per query object queries
    kPreset = 91,                     // the last LOD's item presets (within queries)
};

template <typename T>
T* buf(tdp_ctx* ctx, int slot) { return (T*)ctx->scratch[slot].p; }

// Everything the tuned form's LOD loop (and the FP64 recheck after it) hands
// to its launches.  The loop's launches are a pure function of these bytes, so
// they are also the key of the context's cached CUDA graph of the loop: an
// equal key replays the graph, any difference (a grown scratch buffer, another
// tile, V, the LOD list, the refine configuration) captures it again.
struct LodLoop {
    JoinDev d;
    int nl, li[8], highest_k;
    const float4 *tri1[8], *tri2[8];
    const uint32_t *vt1[8], *vt2[8];
    const float4 *tri1_100, *tri2_100;
    const uint32_t *vt1_100, *vt2_100;
    RefineItem* items;
    int* item_vp;
    float4* res;
    unsigned* counter;
    unsigned long long* dstats;
    int num_sms, cfg[8], hlevel, any_knn, any_within, K, knn, recheck;
    int64_t V;
    float tau;
    int* rankst;
    double *vexact, *res64, *pexact;
    // within queries with LOD 100 last: each last-LOD item's preset (its
    // query's distance plus the FP32 error band), so that the refine drops the
    // items and triangle pairs that cannot come within it; NULL otherwise
    float* preset;
    cudaEvent_t ev[16];
    LazyTile lz1, lz2;  // attached tiles: fetch each LOD's voxels before its refine
    cudaStream_t side;  // attached tiles: the next LOD's prefetch runs here
    cudaEvent_t pf[16];
};

// Enqueue the loop on s.  While s is being captured, the per-LOD timing events
// become event-record nodes of the graph (cudaEventRecordExternal), so that
// a replay still times every refine launch.
int enqueue_lod_loop(tdp_ctx* ctx, const LodLoop& L, cudaStream_t s, bool capturing) {
#define CUL(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)
    auto rec = [&](cudaEvent_t e) {
        return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
    };
    unsigned* cnt_items = L.counter + 8;     // [0] items, [2..3] tri-pair sum (u64)
    unsigned* lod_counts = L.counter + 24;   // per-LOD item counts
    unsigned* cnt_recheck = L.counter + 32;  // pairs left for the FP64 recheck
    const int V = (int)L.V;
    CUL(cudaMemsetAsync(L.counter + 8, 0, 26 * sizeof(unsigned), s));
    CUL(cudaMemsetAsync(L.dstats, 0, 8, s));
    // Attached tiles: once LOD k's own voxels are fetched, a second stream
    // prefetches LOD k+1 for every live voxel pair of an undecided object pair
    // (a superset of LOD k+1's items) while LOD k refines; LOD k+1's fetch
    // waits for it first and then copies only what the prefetch missed.
    const bool prefetch = (L.lz1.on || L.lz2.on) && L.side;
    for (int k = 0; k < L.nl; ++k) {
        const int highest = k == L.highest_k;
        float* preset = highest ? L.preset : nullptr;
        CUL(cudaMemsetAsync(cnt_items, 0, 4, s));
        CUL(launch_build_items(L.d, L.vt1[k], L.vt2[k], L.items, L.item_vp, cnt_items, s, preset, L.tau));
        if (prefetch && k > 0) CUL(cudaStreamWaitEvent(s, L.pf[2 * (k - 1) + 1], 0));
        CUL(launch_fetch_items(L.items, cnt_items, 0, L.li[k], L.lz1, L.lz2, L.num_sms, s));
        if (prefetch && k + 1 < L.nl) {
            CUL(cudaEventRecord(L.pf[2 * k], s));
            CUL(cudaStreamWaitEvent(L.side, L.pf[2 * k], 0));
            CUL(launch_prefetch_pairs(L.d.valive, L.d.vpair, L.d.pstat, L.d.vpa, L.d.vpb, L.V, L.li[k + 1], L.lz1,
                                      L.lz2, L.num_sms, L.side));
            CUL(cudaEventRecord(L.pf[2 * k + 1], L.side));
        }
        CUL(cudaMemcpyAsync(lod_counts + k, cnt_items, 4, cudaMemcpyDeviceToDevice, s));
        CUL(rec(L.ev[2 * k]));
        CUL(launch_refine_tuned(L.tri1[k], L.tri2[k], L.items, V, L.res, L.counter, L.dstats, L.num_sms, L.cfg[k], s,
                                cnt_items, preset));
        CUL(rec(L.ev[2 * k + 1]));
        CUL(launch_apply_results(L.d, L.res, L.item_vp, V, highest, L.hlevel, L.li[k], k, s, cnt_items, preset));
        // the within decision is taken inside the pair update; the kNN rank
        // reads every candidate of a query and stays its own launch
        CUL(launch_pair_update(L.d, k, 1, s, L.any_within ? 1 : 0, L.tau));
        if (L.any_knn) CUL(launch_knn_rank(L.d, L.K, 1, L.rankst, s));
    }
    if (L.recheck) {
        CUL(launch_count_status(L.d, cnt_recheck, s));
        CUL(cudaMemsetAsync(cnt_items, 0, 4, s));
        CUL(launch_recheck_items(L.d, L.vt1_100, L.vt2_100, L.items, L.item_vp, L.vexact, cnt_items, s));
        CUL(launch_fetch_items(L.items, cnt_items, 0, kNumLods - 1, L.lz1, L.lz2, L.num_sms, s));
        CUL(launch_refine_f64(L.tri1_100, L.tri2_100, L.items, V, L.res64, s, cnt_items));
        CUL(launch_recheck_finish(L.d, L.res64, L.item_vp, V, L.vexact, L.pexact, L.knn, L.K, L.tau, s, cnt_items));
    }
#undef CUL
    return TDP_OK;
}

// Run the loop directly or through the context's graph (tdp_set_lod_graph).
// *how: 0 launched directly, 1 replayed the cached graph, 2 captured it now.
int run_lod_loop(tdp_ctx* ctx, const LodLoop& L, cudaStream_t s, long* how) {
    *how = 0;
    const unsigned char* kb = reinterpret_cast<const unsigned char*>(&L);
    auto equal = [&](const std::vector<unsigned char>& v) {
        return v.size() == sizeof(LodLoop) && std::memcmp(v.data(), kb, sizeof(LodLoop)) == 0;
    };
    const int mode = ctx->lod_graph_mode;
    if (mode == TDP_LOD_GRAPH_OFF) return enqueue_lod_loop(ctx, L, s, false);
    if (ctx->lod_graph && equal(ctx->lod_key)) {
        *how = 1;
        const cudaError_t e = cudaGraphLaunch(ctx->lod_graph, s);
        return e == cudaSuccess ? TDP_OK : fail(ctx, TDP_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    }
    if (mode == TDP_LOD_GRAPH_AUTO && !equal(ctx->lod_seen)) {
        // a key seen for the first time runs directly: one-off joins (a served
        // batch) never pay for a capture
        ctx->lod_seen.assign(kb, kb + sizeof(LodLoop));
        return enqueue_lod_loop(ctx, L, s, false);
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    const int rc = enqueue_lod_loop(ctx, L, s, true);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (rc != TDP_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc != TDP_OK ? rc : fail(ctx, TDP_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    }
    ctx->lod_key.clear();
    if (ctx->lod_graph) {
        // same launch sequence with other arguments: update the executable in place
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ctx->lod_graph, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(ctx->lod_graph);
            ctx->lod_graph = nullptr;
        }
    }
    if (!ctx->lod_graph) {
        e = cudaGraphInstantiate(&ctx->lod_graph, g, 0);
        if (e != cudaSuccess) {
            ctx->lod_graph = nullptr;
            cudaGraphDestroy(g);
            return fail(ctx, TDP_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        }
    }
    cudaGraphDestroy(g);
    ctx->lod_key.assign(kb, kb + sizeof(LodLoop));
    *how = 2;
    e = cudaGraphLaunch(ctx->lod_graph, s);
    return e == cudaSuccess ? TDP_OK : fail(ctx, TDP_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
}

}  // namespace
}  // namespace tdp

using namespace tdp;

extern "C" {

void tdp_join_default_params(tdp_join_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->query = TDP_QUERY_NN;
    p->knn = 1;
    p->within_dist = 1000.f;
    p->n_lods = 0;
    p->hausdorff_level = 2;
    p->form = TDP_FORM_TUNED;
    p->exact_distances = 0;
    p->query_begin = 0;
    p->query_end = -1;
}

int tdp_join(tdp_ctx* ctx, const tdp_tile* t1, const tdp_tile* t2, const tdp_join_params* prm, tdp_result** out) {
    if (!ctx || !t1 || !prm || !out) return TDP_ERR_ARG;
    *out = nullptr;
    const bool self = (t2 == nullptr || t2 == t1);
    if (!t2) t2 = t1;
    const bool knn = prm->query == TDP_QUERY_NN;
    const bool isect = prm->query == TDP_QUERY_INTERSECT;
    // an intersect join takes the decisions of a within join at distance 0
    const float within_dist = isect ? 0.f : prm->within_dist;
    const bool mixed = prm->obj_knn != nullptr;  // per query object queries (a batch of requests)
    bool any_knn = knn, any_within = !knn;
    if (mixed) {
        if (!prm->obj_within) return fail(ctx, TDP_ERR_ARG, "obj_knn given without obj_within");
        any_knn = any_within = false;
        for (long i = 0; i < t1->n_obj; ++i) {
            if (prm->obj_knn[i] < 0) return fail(ctx, TDP_ERR_ARG, "obj_knn must be >= 0");
            if (prm->obj_knn[i] == 0 && !(prm->obj_within[i] >= 0.f))
                return fail(ctx, TDP_ERR_ARG, "obj_within must be >= 0 for within objects");
            (prm->obj_knn[i] > 0 ? any_knn : any_within) = true;
        }
    } else {
        if (!knn && !isect && prm->query != TDP_QUERY_WITHIN)
            return fail(ctx, TDP_ERR_ARG, "query must be nn, within or intersect");
        if (knn && prm->knn < 1) return fail(ctx, TDP_ERR_ARG, "knn must be >= 1");
    }
    if (prm->hausdorff_level < 0 || prm->hausdorff_level > 2) return fail(ctx, TDP_ERR_ARG, "hausdorff_level must be 0, 1 or 2");
    // a shard of a join split over GPUs: only tile-1 objects [q_begin, q_end) are queries
    const long q_begin = prm->query_begin, q_end = prm->query_end < 0 ? t1->n_obj : prm->query_end;
    if (q_begin < 0 || q_begin > q_end || q_end > t1->n_obj)
        return fail(ctx, TDP_ERR_ARG, "query range [" + std::to_string(prm->query_begin) + ", " +
                                          std::to_string(prm->query_end) + ") is not inside tile 1's " +
                                          std::to_string(t1->n_obj) + " objects");
    if (prm->form != TDP_FORM_PLAIN && prm->form != TDP_FORM_TUNED) return fail(ctx, TDP_ERR_ARG, "unknown form");
    if (t1->device != ctx->device || t2->device != ctx->device) return fail(ctx, TDP_ERR_ARG, "tile lives on another device");
    const bool tuned = prm->form == TDP_FORM_TUNED;
    std::vector<int> lods;
    if (prm->n_lods <= 0) lods.assign(kLods, kLods + kNumLods);
    else {
        if (prm->n_lods > 8) return fail(ctx, TDP_ERR_ARG, "at most 8 LODs");
        lods.assign(prm->lods, prm->lods + prm->n_lods);
    }
    std::sort(lods.begin(), lods.end());
    lods.erase(std::unique(lods.begin(), lods.end()), lods.end());
    for (int l : lods)
        if (lod_index(l) < 0) return fail(ctx, TDP_ERR_ARG, "LOD " + std::to_string(l) + " not in the tile (20,40,60,80,100)");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    LastStats st;
    if (cudaEventRecord(ctx->ev[0], s) != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, "event record failed");

    // ---- 1. object candidates ----
    // The tuned form generates them on the GPU (csrc/cand_kernels.cu; a kNN
    // ring search that overflows its shared-memory buffer is redone there with
    // a global one).  The plain form keeps the reference's arrangement, where
    // the host builds the candidate lists (its OpenMP octree queries,
    // KNNJoin.cpp:552-573), with the host grid of src/index.  Both give the
    // same set and order.
    int rc;
#define ENS(slot, bytes) do { if ((rc = ensure(ctx, ctx->scratch[slot], (bytes)))) return rc; } while (0)
#define CU(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)
    std::vector<int64_t> qoff;
    std::vector<int32_t> ids, pq;
    long P = 0;
    bool on_device = false;
    const auto c0 = std::chrono::steady_clock::now();
    const int* dqk = nullptr;
    const float* dqtau = nullptr;
    if (mixed) {
        const size_t n1z = (size_t)std::max<long>(t1->n_obj, 1);
        ENS(kQk, n1z * 4);
        ENS(kQtau, n1z * 4);
        dqk = buf<int>(ctx, kQk);
        dqtau = buf<float>(ctx, kQtau);
        CU(cudaMemcpyAsync((void*)dqk, prm->obj_knn, t1->n_obj * 4, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync((void*)dqtau, prm->obj_within, t1->n_obj * 4, cudaMemcpyHostToDevice, s));
    }
    if (tuned) {
        if ((rc = device_candidates(ctx, t1, t2, self, knn, knn ? prm->knn : 0, within_dist, ctx->scratch[kPq],
                                    ctx->scratch[kPt], ctx->scratch[kQoff], P, st.candidate_redone, dqk, dqtau,
                                    isect, q_begin, q_end)))
            return rc;
        on_device = true;
        st.candidates_on_device = 1;
    }
    if (!on_device) {
        CandidateQuery cq{t1->host.obj_box.data(), t1->host.obj_xf.data(), t1->n_obj, t2->host.obj_box.data(),
                          t2->host.obj_xf.data(), t2->n_obj, self, knn, knn ? prm->knn : 0, within_dist, 0,
                          prm->obj_knn, prm->obj_within, isect, q_begin, q_end};
        generate_candidates(cq, qoff, ids);
        P = (long)ids.size();
        if (P >= (1L << 31) - 1) return fail(ctx, TDP_ERR_ARG, "too many candidate pairs");
        pq.resize(P);
        for (long i = 0; i < t1->n_obj; ++i)
            for (int64_t k = qoff[i]; k < qoff[i + 1]; ++k) pq[k] = (int32_t)i;
    }
    st.candidates_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - c0).count();

    const size_t Pz = (size_t)std::max<long>(P, 1);
    ENS(kPq, Pz * 4); ENS(kPt, Pz * 4); ENS(kQoff, (t1->n_obj + 1) * 8);
    ENS(kPmn, Pz * 4); ENS(kPmx, Pz * 4); ENS(kPerr, Pz * 4); ENS(kPstat, Pz);
    ENS(kPvp, (Pz + 1) * 8); ENS(kQconf, (t1->n_obj + 1) * 4); ENS(kCnt, (Pz + 1) * 8); ENS(kRankSt, Pz * 4);
    ENS(kOutQ, Pz * 4); ENS(kOutT, Pz * 4); ENS(kOutD, Pz * 4);

    JoinDev d;
    std::memset(&d, 0, sizeof d);  // padding too: the LOD loop's graph key holds these bytes
    d.vox1 = t1->vox; d.ovox1 = t1->obj_vox; d.vox2 = t2->vox; d.ovox2 = t2->obj_vox;
    d.ohd1 = t1->obj_hd; d.ophd1 = t1->obj_phd; d.ohd2 = t2->obj_hd; d.ophd2 = t2->obj_phd;
    d.P = (int)P;
    d.pq = buf<int>(ctx, kPq); d.pt = buf<int>(ctx, kPt);
    d.pmn = buf<float>(ctx, kPmn); d.pmx = buf<float>(ctx, kPmx); d.perr = buf<float>(ctx, kPerr);
    d.pstat = buf<uint8_t>(ctx, kPstat); d.pvp = buf<int64_t>(ctx, kPvp);
    d.N1 = (int)t1->n_obj; d.qoff = buf<int64_t>(ctx, kQoff); d.qconf = buf<int>(ctx, kQconf);
    d.qk = dqk; d.qtau = dqtau; d.isect = isect ? 1 : 0;
    d.early_tau = (tuned && !knn && !mixed && !isect) ? within_dist : -1.f;
    d.early_mixed = (tuned && mixed) ? 1 : 0;

    unsigned* cnt_items = ctx->d_counter + 8;    // [0] items, [2..3] tri-pair sum (u64)
    unsigned* cnt_status = ctx->d_counter + 16;  // undecided, reported
    unsigned* cnt_collect = ctx->d_counter + 20;

    CU(cudaEventRecord(ctx->ev[5], s));
    if (!on_device) {
        if (P > 0) {
            CU(cudaMemcpyAsync((void*)d.pq, pq.data(), P * 4, cudaMemcpyHostToDevice, s));
            CU(cudaMemcpyAsync((void*)d.pt, ids.data(), P * 4, cudaMemcpyHostToDevice, s));
        }
        CU(cudaMemcpyAsync((void*)d.qoff, qoff.data(), qoff.size() * 8, cudaMemcpyHostToDevice, s));
    }
    CU(cudaMemsetAsync(d.qconf, 0, t1->n_obj * 4, s));
    CU(cudaMemsetAsync(ctx->d_stats + 1, 0, 8, s));
    // attached tiles: voxels fetched on demand, bytes counted per join
    LazyTile lz1 = lazy_view(t1), lz2 = lazy_view(t2);
    unsigned long long* fetch_ctr = ctx->d_stats + 8;
    if (lz1.on) lz1.bytes = fetch_ctr;
    if (lz2.on) lz2.bytes = fetch_ctr;
    CU(cudaMemsetAsync(fetch_ctr, 0, 8, s));
    d.stat_vp = ctx->d_stats + 1;
    long launches = 0;

    // ---- 2. filter ----
    CU(launch_pair_bounds(d, s)); ++launches;
    if (any_knn) { CU(launch_knn_rank(d, prm->knn, tuned, buf<int>(ctx, kRankSt), s)); }
    if (any_within) { CU(launch_within_decide(d, within_dist, tuned, s)); }
    ++launches;
    int64_t* cnt = buf<int64_t>(ctx, kCnt);
    CU(cudaMemsetAsync(cnt + P, 0, 8, s));
    CU(launch_count_vps(d, !knn, within_dist, tuned, cnt, s)); ++launches;
    size_t tmp_bytes = 0;
    CU(scan_counts(cnt, d.pvp, (int)P, nullptr, tmp_bytes, s));
    ENS(kScanTmp, tmp_bytes + 16);
    CU(scan_counts(cnt, d.pvp, (int)P, ctx->scratch[kScanTmp].p, tmp_bytes, s)); ++launches;
    int64_t V = 0;
    CU(cudaMemcpyAsync(&V, d.pvp + P, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const size_t Vz = (size_t)std::max<int64_t>(V, 1);
    ENS(kVpa, Vz * 4); ENS(kVpb, Vz * 4); ENS(kVpair, Vz * 4); ENS(kVmn, Vz * 4); ENS(kVmx, Vz * 4);
    ENS(kVerr, Vz * 4); ENS(kValive, Vz); ENS(kVupd, Vz * 4);
    ENS(kItems, Vz * sizeof(RefineItem)); ENS(kItemVp, Vz * 4); ENS(kRes, Vz * sizeof(float4));
    d.V = V;
    d.vpa = buf<int>(ctx, kVpa); d.vpb = buf<int>(ctx, kVpb); d.vpair = buf<int>(ctx, kVpair);
    d.vmn = buf<float>(ctx, kVmn); d.vmx = buf<float>(ctx, kVmx); d.verr = buf<float>(ctx, kVerr);
    d.valive = buf<uint8_t>(ctx, kValive); d.vupd = buf<int>(ctx, kVupd);
    CU(launch_write_vps(d, !knn, within_dist, tuned, s)); ++launches;
    CU(cudaEventRecord(ctx->ev[1], s));
    st.filter_pairs = P;

    // ---- 3. LOD loop ----
    RefineItem* items = buf<RefineItem>(ctx, kItems);
    int* item_vp = buf<int>(ctx, kItemVp);
    float4* res = buf<float4>(ctx, kRes);
    double refine_ms = 0;
    unsigned long long full_total = 0;
    double tri_total = 0;
    long refine_items = 0;
    unsigned undecided = 0;
    long syncs = 2;  // candidates upload + voxel-pair count
    if (!tuned) {
        // plain form: the host reads every count, like the reference's chunk loop
        for (size_t k = 0; k < lods.size() && V > 0; ++k) {
            const int li = lod_index(lods[k]);
            const bool highest = (k + 1 == lods.size());
            CU(cudaMemsetAsync(ctx->d_counter + 8, 0, 32, s));
            CU(launch_build_items(d, t1->vtri[li], t2->vtri[li], items, item_vp, cnt_items, s)); ++launches;
            unsigned hc[4];
            CU(cudaMemcpyAsync(hc, cnt_items, 16, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s)); ++syncs;
            const int W = (int)hc[0];
            unsigned long long trip;
            std::memcpy(&trip, &hc[2], 8);
            tri_total += (double)trip;
            refine_items += W;
            if (W > 0) {
                CU(launch_fetch_items(items, nullptr, W, li, lz1, lz2, ctx->num_sms, s));
                if (lz1.on || lz2.on) launches += 2;
                CU(cudaEventRecord(ctx->ev[2], s));
                CU(launch_refine_plain(t1->tri[li], t2->tri[li], items, W, res, s));
                CU(cudaEventRecord(ctx->ev[3], s));
                ++launches;
                st.refine_launches++;
                CU(launch_apply_results(d, res, item_vp, W, highest, prm->hausdorff_level, li, (int)k, s)); ++launches;
            }
            CU(launch_pair_update(d, (int)k, 0, s)); ++launches;
            if (any_knn) CU(launch_knn_rank(d, prm->knn, 0, buf<int>(ctx, kRankSt), s));
            if (any_within) CU(launch_within_decide(d, within_dist, 0, s));
            ++launches;
            CU(cudaMemsetAsync(cnt_status, 0, 8, s));
            CU(launch_count_status(d, cnt_status, s)); ++launches;
            unsigned sc[2];
            CU(cudaMemcpyAsync(sc, cnt_status, 8, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s)); ++syncs;
            if (W > 0) {
                float ms = 0;
                cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
                refine_ms += ms;
                full_total += trip;
            }
            undecided = sc[0];
            if (sc[0] == 0) break;
        }
    } else if (V > 0) {
        // tuned form: every count stays on the device, so the whole loop (and
        // the FP64 recheck) is enqueued without a host round trip; kernels with
        // nothing left to do exit at once
        ENS(kVexact, Vz * 8); ENS(kPexact, Pz * 8); ENS(kRes64, Vz * 8);
        const bool presets = any_within && !isect && lods.back() == 100;
        if (presets) ENS(kPreset, Vz * 4);
        // 3b. after LOD 100, the FP64 recheck of pairs whose FP32 ranges
        // stayed inside their error band
        LodLoop L;
        std::memset(&L, 0, sizeof L);  // padding included: the bytes are the graph's key
        L.d = d;
        L.nl = (int)lods.size();
        L.highest_k = L.nl - 1;
        for (int k = 0; k < L.nl; ++k) {
            const int li = lod_index(lods[k]);
            L.li[k] = li;
            L.tri1[k] = t1->tri[li]; L.tri2[k] = t2->tri[li];
            L.vt1[k] = t1->vtri[li]; L.vt2[k] = t2->vtri[li];
            L.ev[2 * k] = ctx->lod_ev[2 * k];
            L.ev[2 * k + 1] = ctx->lod_ev[2 * k + 1];
        }
        L.recheck = lods.back() == 100;
        L.tri1_100 = t1->tri[4]; L.tri2_100 = t2->tri[4];
        L.vt1_100 = t1->vtri[4]; L.vt2_100 = t2->vtri[4];
        L.items = items; L.item_vp = item_vp; L.res = res;
        L.counter = ctx->d_counter; L.dstats = ctx->d_stats;
        L.num_sms = ctx->num_sms; L.hlevel = prm->hausdorff_level;
        for (int k = 0; k < L.nl; ++k) L.cfg[k] = ctx->lod_cfg[L.li[k]] >= 0 ? ctx->lod_cfg[L.li[k]] : ctx->tuned_cfg;
        L.any_knn = any_knn; L.any_within = any_within; L.K = prm->knn; L.knn = knn;
        L.V = V; L.tau = within_dist;
        L.rankst = buf<int>(ctx, kRankSt);
        L.vexact = buf<double>(ctx, kVexact); L.res64 = buf<double>(ctx, kRes64); L.pexact = buf<double>(ctx, kPexact);
        L.lz1 = lz1; L.lz2 = lz2;
        L.preset = presets ? buf<float>(ctx, kPreset) : nullptr;
        L.side = ctx->side;
        for (int k = 0; k < 16; ++k) L.pf[k] = ctx->pf_ev[k];
        if ((rc = run_lod_loop(ctx, L, s, &st.lod_graph))) return rc;
        {   // per LOD: items, refine, apply, pair update (with the within decision),
            // the kNN rank; on attached tiles the fetch and the next LOD's prefetch
            const bool attached = L.lz1.on || L.lz2.on;
            // (a fetch or a prefetch is a mark launch and a copy launch)
            launches += (4 + (L.any_knn ? 1 : 0) + (attached ? 2 : 0)) * L.nl +
                        (attached && L.side ? 2 * (L.nl - 1) : 0) +
                        (L.recheck ? (knn ? 5 : 4) + (attached ? 2 : 0) : 0);
        }
        st.refine_launches += L.nl;
    }

    // ---- 4. exact LOD-100 distances of the reported pairs (optional) ----
    const bool exact = prm->exact_distances != 0;
    double* pex = nullptr;
    ExactInfo xi;
    if (exact) {
        ENS(kPexOut, Pz * 8);
        ENS(kOutD64, Pz * 8);
        pex = buf<double>(ctx, kPexOut);
        CU(cudaEventRecord(ctx->ev[6], s));
        if ((rc = exact_distances(ctx, d, t1, t2, prm->hausdorff_level == 2, pex, xi, lz1, lz2))) return rc;
        CU(cudaEventRecord(ctx->ev[7], s));
        launches += xi.launches;
        syncs += 2;
    }

    // ---- 5. results ----
    CU(cudaMemsetAsync(cnt_collect, 0, 4, s));
    {
        size_t sort_bytes = 0;
        CU(collect_sort_bytes(P, t1->n_obj, t2->n_obj, sort_bytes));
        ENS(kKeyA, Pz * 8); ENS(kKeyB, Pz * 8); ENS(kValA, Pz * 4); ENS(kValB, Pz * 4);
        ENS(kScanTmp, sort_bytes + 16);
        unsigned long long* keys[2] = {buf<unsigned long long>(ctx, kKeyA), buf<unsigned long long>(ctx, kKeyB)};
        int* vals[2] = {buf<int>(ctx, kValA), buf<int>(ctx, kValB)};
        CU(launch_collect(d, t2->n_obj, keys, vals, ctx->scratch[kScanTmp].p, sort_bytes, cnt_collect, pex,
                          buf<int>(ctx, kOutQ), buf<int>(ctx, kOutT), buf<float>(ctx, kOutD),
                          exact ? buf<double>(ctx, kOutD64) : nullptr, s));
        launches += 2;
    }
    CU(cudaEventRecord(ctx->ev[4], s));
    unsigned nres = 0;
    unsigned tc[32] = {0};
    unsigned long long fe = 0;
    CU(cudaMemcpyAsync(&nres, cnt_collect, 4, cudaMemcpyDeviceToHost, s));
    unsigned long long fvp = 0, fetched = 0;
    CU(cudaMemcpyAsync(&fvp, ctx->d_stats + 1, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&fetched, fetch_ctr, 8, cudaMemcpyDeviceToHost, s));
    if (tuned && V > 0) {
        CU(cudaMemcpyAsync(tc, ctx->d_counter + 8, 32 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(&fe, ctx->d_stats, 8, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    ++syncs;
    st.filter_voxel_pairs = (double)fvp;
    st.fetch_bytes = (double)fetched;
    if (tuned && V > 0) {
        unsigned long long trip;
        std::memcpy(&trip, &tc[2], 8);  // d_counter[10..11]
        tri_total = (double)trip;
        for (size_t k = 0; k < lods.size(); ++k) {
            refine_items += tc[16 + k];     // d_counter[24 + k]
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->lod_ev[2 * k], ctx->lod_ev[2 * k + 1]);
            refine_ms += ms;
            st.refine_ms_lod[lod_index(lods[k])] = ms;
        }
        full_total = fe;
        undecided = lods.back() == 100 ? tc[24] : 0;  // d_counter[32]
        st.recheck_pairs = undecided;
    }
    // rows were sorted by (query, result id) on the device
    tdp_result* R = new tdp_result();
    if (nres) {
        // through a page-locked staging buffer: a fast copy, then one pass
        // into the result (no zero-fill of the vectors first)
        const size_t need = (size_t)nres * (exact ? 20 : 12);
        if (need > ctx->hres_cap) {
            if (ctx->hres) cudaFreeHost(ctx->hres);
            ctx->hres = nullptr;
            ctx->hres_cap = 0;
            const size_t cap = need + need / 4 + 4096;
            if (cudaHostAlloc(&ctx->hres, cap, cudaHostAllocDefault) == cudaSuccess) ctx->hres_cap = cap;
            else ctx->hres = nullptr;
        }
        cudaError_t e;
        if (ctx->hres) {
            uint8_t* h = (uint8_t*)ctx->hres;
            double* h64 = (double*)h;  // 8-byte aligned first
            int* hq = (int*)(h + (exact ? (size_t)nres * 8 : 0));
            int* ht = hq + nres;
            float* hd = (float*)(ht + nres);
            if (exact) cudaMemcpyAsync(h64, buf<double>(ctx, kOutD64), nres * 8, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(hq, buf<int>(ctx, kOutQ), nres * 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(ht, buf<int>(ctx, kOutT), nres * 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(hd, buf<float>(ctx, kOutD), nres * 4, cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            if (e == cudaSuccess) {
                R->q.assign(hq, hq + nres);
                R->t.assign(ht, ht + nres);
                R->d.assign(hd, hd + nres);
                if (exact) R->d64.assign(h64, h64 + nres);
            }
        } else {
            R->q.resize(nres); R->t.resize(nres); R->d.resize(nres);
            cudaMemcpyAsync(R->q.data(), buf<int>(ctx, kOutQ), nres * 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(R->t.data(), buf<int>(ctx, kOutT), nres * 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(R->d.data(), buf<float>(ctx, kOutD), nres * 4, cudaMemcpyDeviceToHost, s);
            if (exact) {
                R->d64.resize(nres);
                cudaMemcpyAsync(R->d64.data(), buf<double>(ctx, kOutD64), nres * 8, cudaMemcpyDeviceToHost, s);
            }
            e = cudaStreamSynchronize(s);
        }
        if (e != cudaSuccess) { delete R; return fail(ctx, TDP_ERR_CUDA, cudaGetErrorString(e)); }
    }
    float f_ms = 0, tot_ms = 0;
    cudaEventElapsedTime(&f_ms, ctx->ev[5], ctx->ev[1]);
    cudaEventElapsedTime(&tot_ms, ctx->ev[0], ctx->ev[4]);
    st.filter_ms = f_ms;
    st.total_ms = tot_ms;
    st.refine_ms = refine_ms;
    st.tri_pairs = tri_total;
    st.full_evals = full_total;
    st.refine_items = refine_items;
    st.kernel_launches = launches;
    st.host_syncs = syncs;
    {
        float lms = 0, xms = 0;
        cudaEventElapsedTime(&lms, ctx->ev[1], ctx->ev[4]);
        if (exact) cudaEventElapsedTime(&xms, ctx->ev[6], ctx->ev[7]);
        st.lod_ms = lms - xms;
        st.exact_ms = xms;
        st.exact_items = xi.items;
        st.exact_f64_items = xi.f64_items;
        st.fp32_max_rel_err = xi.max_rel_err32;
        for (int k = 0; k < 4; ++k) st.exact_phase_ms[k] = xi.phase_ms[k];
        st.exact_full_evals = xi.full_evals;
        st.exact_dropped_items = xi.dropped_items;
        st.exact_below_items = xi.below_items;
    }
    ctx->stats = st;
    *out = R;
#undef ENS
#undef CU
    return TDP_OK;
}

int tdp_autotune(tdp_ctx* ctx, const tdp_tile* t1, const tdp_tile* t2, const tdp_join_params* prm,
                 double* ms_per_config, int* best) {
    if (!ctx || !t1 || !prm) return TDP_ERR_ARG;
    tdp_join_params p = *prm;
    p.form = TDP_FORM_TUNED;
    const int keep = ctx->tuned_cfg;
    int keep_lod[kNumLods];
    std::memcpy(keep_lod, ctx->lod_cfg, sizeof(keep_lod));
    for (int& c : ctx->lod_cfg) c = -1;
    int best_cfg = keep;
    double best_ms = 1e300;
    double lod_best[kNumLods];
    int lod_arg[kNumLods];
    for (int l = 0; l < kNumLods; ++l) { lod_best[l] = 1e300; lod_arg[l] = -1; }
    for (int cfg = 0; cfg < kTunedConfigs; ++cfg) {
        ctx->tuned_cfg = cfg;
        double ms = 0;
        for (int rep = 0; rep < 2; ++rep) {  // one untimed run, then one timed
            tdp_result* r = nullptr;
            const int rc = tdp_join(ctx, t1, t2, &p, &r);
            if (rc != TDP_OK) {
                ctx->tuned_cfg = keep;
                std::memcpy(ctx->lod_cfg, keep_lod, sizeof(keep_lod));
                return rc;
            }
            tdp_result_free(r);
            ms = ctx->stats.refine_ms;
        }
        if (ms_per_config) ms_per_config[cfg] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best_cfg = cfg;
        }
        // the fastest configuration at each LOD the join refined
        for (int l = 0; l < kNumLods; ++l) {
            const double m = ctx->stats.refine_ms_lod[l];
            if (m > 0 && m < lod_best[l]) { lod_best[l] = m; lod_arg[l] = cfg; }
        }
    }
    ctx->tuned_cfg = best_cfg;
    for (int l = 0; l < kNumLods; ++l) ctx->lod_cfg[l] = lod_arg[l];
    if (best) *best = best_cfg;
    return TDP_OK;
}

int tdp_result_count(const tdp_result* r, long* n) {
    if (!r || !n) return TDP_ERR_ARG;
    *n = (long)r->q.size();
    return TDP_OK;
}

int tdp_result_copy_f64(const tdp_result* r, double* dist) {
    if (!r) return TDP_ERR_ARG;
    if (r->d64.size() != r->q.size()) return TDP_ERR_STATE;
    if (dist) std::memcpy(dist, r->d64.data(), r->d64.size() * 8);
    return TDP_OK;
}

int tdp_result_copy(const tdp_result* r, int* qid, int* rid, float* dist) {
    if (!r) return TDP_ERR_ARG;
    const size_t n = r->q.size();
    if (qid) std::memcpy(qid, r->q.data(), n * 4);
    if (rid) std::memcpy(rid, r->t.data(), n * 4);
    if (dist) std::memcpy(dist, r->d.data(), n * 4);
    return TDP_OK;
}

int tdp_result_free(tdp_result* r) {
    if (!r) return TDP_ERR_ARG;
    delete r;
    return TDP_OK;
}

}  // extern "C"
