// ctx.cuh -- the context object behind the C ABI: device, stream, memory budget,
// reusable scratch buffers and the statistics of the last call.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <unordered_map>
#include <map>
#include <vector>
#include "common.cuh"
#include "storage/dt_format.h"
#include "../../include/tdp.h"

namespace tdp {

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
};

// Statistics of the last refine launch / join, filled by the library.
struct LastStats {
    double refine_ms = 0;            // device time of refine kernels (CUDA events)
    double filter_ms = 0;            // device time of filter kernels
    double total_ms = 0;             // device time of the whole call
    unsigned long long full_evals = 0;  // triangle pairs fully evaluated
    double tri_pairs = 0;            // sum of n1*n2 over refined voxel pairs
    long refine_items = 0;           // voxel pairs refined (all LODs)
    long refine_launches = 0;
    long recheck_pairs = 0;          // object pairs recomputed in FP64
    long filter_pairs = 0;           // object pairs through the filter
    double filter_voxel_pairs = 0;   // voxel pairs evaluated by the filter
    long kernel_launches = 0;        // kernels launched by the call
    double candidates_ms = 0;        // host wall time of object candidate generation
    double lod_ms = 0;               // device time of the LOD loop
    long host_syncs = 0;             // host<->device synchronisations in the call
    double exact_ms = 0;             // device time of the exact-distance stage
    long exact_items = 0;            // LOD-100 voxel pairs it refined in FP32
    long exact_f64_items = 0;        // of those, evaluated in FP64
    double fp32_max_rel_err = 0;     // max |FP32 minimum - FP64 distance| / max(distance, 1)
    double fetch_bytes = 0;          // RAW bytes fetched from attached tiles
    double refine_ms_lod[kNumLods] = {0, 0, 0, 0, 0};  // tuned refine time per LOD index
    long lod_graph = 0;              // tuned LOD loop: 0 direct launches, 1 graph replayed, 2 graph captured
    double exact_phase_ms[4] = {0, 0, 0, 0};  // exact stage: upper bounds, candidates, FP32 pass, FP64 pass
    unsigned long long exact_full_evals = 0;   // exact stage: triangle pairs fully evaluated in FP32
    long candidates_on_device = 0;   // 1: object candidates came from the GPU (the tuned form)
    long candidate_redone = 0;       // kNN queries redone with the global ring-search buffer
    long exact_dropped_items = 0;    // exact stage: FP32-pass items dropped by the item-level test
    long exact_below_items = 0;      // exact stage: FP32-pass items below their preset
};

}  // namespace tdp

struct tdp_ctx {
    int device = 0;
    unsigned flags = 0;  // TDP_CTX_* flags given to tdp_ctx_create
    int num_sms = 148;
    size_t budget = 0, in_use = 0, peak = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    cudaEvent_t lod_ev[16] = {};  // refine timing per LOD (tuned loop)
    cudaEvent_t xev[5] = {};      // phases of the exact-distance stage
    cudaStream_t side = nullptr;  // second stream: the next LOD's prefetch (attached tiles)
    cudaEvent_t pf_ev[16] = {};   // fork / join of the prefetches (no timing)
    std::string last_error;
    std::unordered_map<void*, size_t> allocs;
    tdp::Buf scratch[104];  // slots: refine-batch 0-4, tile upload 12-13, join 20-48, candidates 50-59 and 88-90, result sort 60-63, exact distances 64-81 and 84-86, per-object queries 82-83, last-LOD presets 91, GPU attach pass 96-100
    unsigned* d_counter = nullptr;            // work counters (device)
    unsigned long long* d_stats = nullptr;    // device-side statistics
    tdp::LastStats stats;
    int tuned_cfg = 0;  // tuned refine kernel configuration (tdp_set_refine_config / tdp_autotune)
    // per LOD index (20..100): the configuration the autotuner found fastest
    // at that LOD (-1: tuned_cfg); tdp_set_refine_config clears them
    int lod_cfg[tdp::kNumLods] = {-1, -1, -1, -1, -1};
    void* hres = nullptr;  // page-locked staging of join results (grow-only)
    size_t hres_cap = 0;
    // CUDA graph of the tuned form's LOD loop (tdp_set_lod_graph): the
    // executable, the launch arguments it was captured with, and the last
    // arguments launched directly (auto mode captures a key on its second use)
    int lod_graph_mode = TDP_LOD_GRAPH_AUTO;
    cudaGraphExec_t lod_graph = nullptr;
    std::vector<unsigned char> lod_key, lod_seen;
    // idle device blocks of released tiles' triangle arrays, by size, handed
    // back to the next tile of (about) the same size: re-attaching or
    // re-uploading a tile costs no cudaMalloc / cudaFree of tens of GB.  Not
    // counted in in_use; trimmed when an allocation would fail or exceed the
    // budget, and on destroy.
    std::multimap<size_t, void*> block_cache;
    size_t cached_bytes = 0;
    size_t small_cached = 0;  // cached blocks below kCachedBlockMin
    // page-locked staging of tile metadata (grow-only): two buffers taken in
    // turn, each with an event recorded after its last copy, so an attach
    // returns while its copies run and the next attach stages into the other
    void* hstage[2] = {nullptr, nullptr};
    size_t hstage_cap[2] = {0, 0};
    cudaEvent_t hstage_ev[2] = {nullptr, nullptr};
    int hstage_next = 0;
};

namespace tdp {

int fail(tdp_ctx* ctx, int code, const std::string& msg);
cudaError_t dmalloc(tdp_ctx* ctx, void** p, size_t bytes);
void dfree(tdp_ctx* ctx, void* p);
// grow-only scratch buffer; returns TDP_OK or an error status (recorded in ctx)
int ensure(tdp_ctx* ctx, Buf& b, size_t bytes);
// blocks for tile arrays: block_alloc reuses an idle cached block of the
// size (or up to 25 % larger); block_release caches the block (the caller
// has synchronised the context's stream, so the block is idle).  Requests
// below kCachedBlockMin are rounded up to a power of two of at least 256
// bytes, so a small block fits the next request of its class exactly; at
// most kSmallCached small blocks stay cached, further ones are freed.  A
// tile's small arrays (object and voxel offsets of a tile of a thousand
// objects) then cost no cudaMalloc / cudaFree per attach either.
constexpr size_t kCachedBlockMin = (size_t)1 << 20;
constexpr size_t kSmallCached = 512;
cudaError_t block_alloc(tdp_ctx* ctx, void** p, size_t bytes);
void block_release(tdp_ctx* ctx, void* p);
void cache_trim(tdp_ctx* ctx);

enum ScratchSlot {
    kSlotRawData = 0, kSlotRawHd, kSlotTris, kSlotItems, kSlotOut,
};

}  // namespace tdp
