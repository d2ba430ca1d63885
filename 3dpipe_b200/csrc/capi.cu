// capi.cu -- context management and the refine seam of the C ABI (include/tdp.h).
#include <float.h>
#include <algorithm>
#include <string.h>
#include <vector>
#include "ctx.cuh"
#include "refine.cuh"

namespace tdp {

int fail(tdp_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

void cache_trim(tdp_ctx* ctx) {
    for (auto& kv : ctx->block_cache) cudaFree(kv.second);
    ctx->block_cache.clear();
    ctx->cached_bytes = 0;
    ctx->small_cached = 0;
}

cudaError_t dmalloc(tdp_ctx* ctx, void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (ctx->budget && ctx->in_use + bytes > ctx->budget) return cudaErrorMemoryAllocation;
    if (ctx->budget && ctx->in_use + ctx->cached_bytes + bytes > ctx->budget) cache_trim(ctx);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess && !ctx->block_cache.empty()) {  // the cache holds the memory: give it back, retry
        cudaGetLastError();
        cache_trim(ctx);
        e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) { *p = nullptr; return e; }
    ctx->allocs[*p] = bytes;
    ctx->in_use += bytes;
    if (ctx->in_use + ctx->cached_bytes > ctx->peak) ctx->peak = ctx->in_use + ctx->cached_bytes;
    return cudaSuccess;
}

static size_t block_class(size_t bytes) {
    if (bytes >= kCachedBlockMin) return bytes;
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
}

cudaError_t block_alloc(tdp_ctx* ctx, void** p, size_t bytes) {
    *p = nullptr;
    bytes = block_class(bytes == 0 ? 16 : bytes);
    auto it = ctx->block_cache.lower_bound(bytes);
    if (it != ctx->block_cache.end() && it->first <= bytes + bytes / 4) {
        if (ctx->budget && ctx->in_use + it->first > ctx->budget) return cudaErrorMemoryAllocation;
        *p = it->second;
        ctx->allocs[*p] = it->first;
        ctx->in_use += it->first;
        ctx->cached_bytes -= it->first;
        if (it->first < kCachedBlockMin) --ctx->small_cached;
        ctx->block_cache.erase(it);
        return cudaSuccess;
    }
    return dmalloc(ctx, p, bytes);
}

void block_release(tdp_ctx* ctx, void* p) {
    if (!p) return;
    auto it = ctx->allocs.find(p);
    if (it == ctx->allocs.end() || (it->second < kCachedBlockMin && ctx->small_cached >= kSmallCached)) {
        dfree(ctx, p);
        return;
    }
    if (it->second < kCachedBlockMin) ++ctx->small_cached;
    ctx->in_use -= it->second;
    ctx->cached_bytes += it->second;
    ctx->block_cache.emplace(it->second, p);
    ctx->allocs.erase(it);
}

void dfree(tdp_ctx* ctx, void* p) {
    if (!p) return;
    auto it = ctx->allocs.find(p);
    if (it != ctx->allocs.end()) {
        ctx->in_use -= it->second;
        ctx->allocs.erase(it);
    }
    cudaFree(p);
}

int ensure(tdp_ctx* ctx, Buf& b, size_t bytes) {
    if (bytes <= b.cap && b.p) return TDP_OK;
    if (b.p) { dfree(ctx, b.p); b.p = nullptr; b.cap = 0; }
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = dmalloc(ctx, &b.p, want);
    if (e != cudaSuccess) {
        e = dmalloc(ctx, &b.p, bytes);
        if (e != cudaSuccess)
            return fail(ctx, TDP_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                                               (ctx->budget && ctx->in_use + bytes > ctx->budget
                                                    ? std::string("context budget exceeded")
                                                    : std::string(cudaGetErrorString(e))));
        b.cap = bytes;
        return TDP_OK;
    }
    b.cap = want;
    return TDP_OK;
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void fma_probe_kernel(float* out, int iters, float b, float c) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1.2345f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace tdp

using namespace tdp;

extern "C" {

int tdp_ctx_create(int device, size_t budget_bytes, unsigned flags, tdp_ctx** out) {
    if (!out) return TDP_ERR_ARG;
    if (flags & ~(unsigned)TDP_CTX_POISON) return TDP_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return TDP_ERR_NODEV;
    if (device < 0 || device >= n) return TDP_ERR_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TDP_ERR_NODEV;
    if (prop.major != 10) return TDP_ERR_NODEV;  // kernels are built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return TDP_ERR_NODEV;
    tdp_ctx* ctx = new tdp_ctx();
    ctx->device = device;
    ctx->budget = budget_bytes;
    ctx->flags = flags;
    ctx->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return TDP_ERR_CUDA; }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    for (auto& e : ctx->lod_ev) cudaEventCreate(&e);
    for (auto& e : ctx->xev) cudaEventCreate(&e);
    for (auto& e : ctx->pf_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess) {
        tdp_ctx_destroy(ctx);
        return TDP_ERR_CUDA;
    }
    if (dmalloc(ctx, (void**)&ctx->d_counter, 64 * sizeof(unsigned)) != cudaSuccess ||
        dmalloc(ctx, (void**)&ctx->d_stats, 64 * sizeof(unsigned long long)) != cudaSuccess) {
        tdp_ctx_destroy(ctx);
        return TDP_ERR_NOMEM;
    }
    *out = ctx;
    return TDP_OK;
}

int tdp_ctx_destroy(tdp_ctx* ctx) {
    if (!ctx) return TDP_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    std::vector<void*> ptrs;
    for (auto& kv : ctx->allocs) ptrs.push_back(kv.first);
    for (void* p : ptrs) dfree(ctx, p);
    for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->lod_ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->xev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->pf_ev) if (e) cudaEventDestroy(e);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    cache_trim(ctx);
    if (ctx->lod_graph) cudaGraphExecDestroy(ctx->lod_graph);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->hres) cudaFreeHost(ctx->hres);
    for (int k = 0; k < 2; ++k) {
        if (ctx->hstage[k]) cudaFreeHost(ctx->hstage[k]);
        if (ctx->hstage_ev[k]) cudaEventDestroy(ctx->hstage_ev[k]);
    }
    delete ctx;
    return TDP_OK;
}

const char* tdp_last_error(const tdp_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int tdp_last_stats(const tdp_ctx* ctx, tdp_stats* o) {
    if (!ctx || !o) return TDP_ERR_ARG;
    const LastStats& s = ctx->stats;
    o->refine_ms = s.refine_ms;
    o->filter_ms = s.filter_ms;
    o->total_ms = s.total_ms;
    o->full_evals = s.full_evals;
    o->tri_pairs = s.tri_pairs;
    o->refine_items = s.refine_items;
    o->refine_launches = s.refine_launches;
    o->recheck_pairs = s.recheck_pairs;
    o->filter_pairs = s.filter_pairs;
    o->filter_voxel_pairs = s.filter_voxel_pairs;
    o->kernel_launches = s.kernel_launches;
    o->candidates_ms = s.candidates_ms;
    o->lod_ms = s.lod_ms;
    o->host_syncs = s.host_syncs;
    o->exact_ms = s.exact_ms;
    o->exact_items = s.exact_items;
    o->exact_f64_items = s.exact_f64_items;
    o->fp32_max_rel_err = s.fp32_max_rel_err;
    o->fetch_bytes = s.fetch_bytes;
    for (int l = 0; l < tdp::kNumLods; ++l) o->refine_ms_lod[l] = s.refine_ms_lod[l];
    o->lod_graph = s.lod_graph;
    for (int k = 0; k < 4; ++k) o->exact_phase_ms[k] = s.exact_phase_ms[k];
    o->exact_full_evals = s.exact_full_evals;
    o->candidates_on_device = s.candidates_on_device;
    o->candidate_redone = s.candidate_redone;
    o->exact_dropped_items = s.exact_dropped_items;
    o->exact_below_items = s.exact_below_items;
    return TDP_OK;
}

int tdp_set_lod_graph(tdp_ctx* ctx, int mode) {
    if (!ctx) return TDP_ERR_ARG;
    if (mode < TDP_LOD_GRAPH_OFF || mode > TDP_LOD_GRAPH_ALWAYS) return fail(ctx, TDP_ERR_ARG, "LOD graph mode must be 0, 1 or 2");
    ctx->lod_graph_mode = mode;
    return TDP_OK;
}

int tdp_fp32_peak(tdp_ctx* ctx, double* tflops) {
    if (!ctx || !tflops) return TDP_ERR_ARG;
    cudaSetDevice(ctx->device);
    const int blocks = ctx->num_sms * 8, threads = 256, iters = 1 << 15;
    float* out = (float*)ctx->d_stats;
    double best = 0;
    for (int rep = 0; rep < 6; ++rep) {
        TDP_CUDA_TRY(cudaEventRecord(ctx->ev[6], ctx->stream));
        fma_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters, 0.999f, 1e-3f);
        TDP_CUDA_TRY(cudaGetLastError());
        TDP_CUDA_TRY(cudaEventRecord(ctx->ev[7], ctx->stream));
        TDP_CUDA_TRY(cudaEventSynchronize(ctx->ev[7]));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[6], ctx->ev[7]);
        const double fl = 2.0 * 8.0 * iters * (double)blocks * threads;
        if (rep > 0 && ms > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
    }
    *tflops = best;
    return TDP_OK;
}

int tdp_refine_config_count(void) { return tdp::kTunedConfigs; }

int tdp_refine_config_info(int cfg, int* chunk_a, int* ctas_per_sm) {
    if (cfg < 0 || cfg >= tdp::kTunedConfigs) return TDP_ERR_ARG;
    const tdp::TunedConfig c = tdp::tuned_config(cfg);
    if (chunk_a) *chunk_a = c.chunk_a;
    if (ctas_per_sm) *ctas_per_sm = c.ctas_per_sm;
    return TDP_OK;
}

int tdp_set_refine_config(tdp_ctx* ctx, int cfg) {
    if (!ctx) return TDP_ERR_ARG;
    if (cfg < 0 || cfg >= tdp::kTunedConfigs)
        return tdp::fail(ctx, TDP_ERR_ARG, "refine configuration " + std::to_string(cfg) + " out of range");
    ctx->tuned_cfg = cfg;
    for (int& c : ctx->lod_cfg) c = -1;
    return TDP_OK;
}

int tdp_get_refine_config_lod(const tdp_ctx* ctx, int lod, int* cfg) {
    if (!ctx || !cfg) return TDP_ERR_ARG;
    const int li = tdp::lod_index(lod);
    if (li < 0) return TDP_ERR_ARG;
    *cfg = ctx->lod_cfg[li] >= 0 ? ctx->lod_cfg[li] : ctx->tuned_cfg;
    return TDP_OK;
}

int tdp_get_refine_config(const tdp_ctx* ctx, int* cfg) {
    if (!ctx || !cfg) return TDP_ERR_ARG;
    *cfg = ctx->tuned_cfg;
    return TDP_OK;
}

void* tdp_ctx_stream(const tdp_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int tdp_ctx_memory(const tdp_ctx* ctx, size_t* in_use, size_t* peak) {
    if (!ctx) return TDP_ERR_ARG;
    if (in_use) *in_use = ctx->in_use + ctx->cached_bytes;  // idle cached tile blocks are held too
    if (peak) *peak = ctx->peak;
    return TDP_OK;
}

int tdp_refine_batch(tdp_ctx* ctx, const float* data, const float* hausdorff, size_t element_num,
                     const size_t* offset_size, uint32_t pair_num, int form, float* out) {
    if (!ctx) return TDP_ERR_ARG;
    if (pair_num == 0) return TDP_OK;
    if (!data || !offset_size || !out) return fail(ctx, TDP_ERR_ARG, "null buffer");
    if (form != TDP_FORM_PLAIN && form != TDP_FORM_TUNED) return fail(ctx, TDP_ERR_ARG, "unknown form");
    if (element_num == 0 || element_num > 0xffffffffull) return fail(ctx, TDP_ERR_ARG, "element_num out of range");
    cudaSetDevice(ctx->device);
    std::vector<RefineItem> items(pair_num);
    double tri_pairs = 0;
    for (uint32_t i = 0; i < pair_num; ++i) {
        size_t o1 = offset_size[4 * i], n1 = offset_size[4 * i + 1];
        size_t o2 = offset_size[4 * i + 2], n2 = offset_size[4 * i + 3];
        if (o1 + n1 > element_num || o2 + n2 > element_num || o1 + n1 < o1 || o2 + n2 < o2)
            return fail(ctx, TDP_ERR_ARG, "offset_size entry " + std::to_string(i) + " out of range");
        items[i] = RefineItem{(uint32_t)o1, (uint32_t)n1, (uint32_t)o2, (uint32_t)n2};
        tri_pairs += (double)n1 * (double)n2;
    }
    int rc;
    if ((rc = ensure(ctx, ctx->scratch[kSlotRawData], element_num * 9 * sizeof(float)))) return rc;
    if (hausdorff && (rc = ensure(ctx, ctx->scratch[kSlotRawHd], element_num * 2 * sizeof(float)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kSlotTris], element_num * kTriF4 * sizeof(float4)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kSlotItems], pair_num * sizeof(RefineItem)))) return rc;
    if ((rc = ensure(ctx, ctx->scratch[kSlotOut], pair_num * sizeof(float4)))) return rc;
    float* d_data = (float*)ctx->scratch[kSlotRawData].p;
    float* d_hd = hausdorff ? (float*)ctx->scratch[kSlotRawHd].p : nullptr;
    float4* d_tri = (float4*)ctx->scratch[kSlotTris].p;
    RefineItem* d_items = (RefineItem*)ctx->scratch[kSlotItems].p;
    float4* d_out = (float4*)ctx->scratch[kSlotOut].p;
    cudaStream_t s = ctx->stream;
    TDP_CUDA_TRY(cudaMemcpyAsync(d_data, data, element_num * 9 * sizeof(float), cudaMemcpyHostToDevice, s));
    if (d_hd) TDP_CUDA_TRY(cudaMemcpyAsync(d_hd, hausdorff, element_num * 2 * sizeof(float), cudaMemcpyHostToDevice, s));
    TDP_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), pair_num * sizeof(RefineItem), cudaMemcpyHostToDevice, s));
    TDP_CUDA_TRY(launch_pack_triangles(d_data, d_hd, element_num, d_tri, s));
    TDP_CUDA_TRY(cudaMemsetAsync(ctx->d_stats, 0, sizeof(unsigned long long), s));
    TDP_CUDA_TRY(cudaEventRecord(ctx->ev[0], s));
    if (form == TDP_FORM_PLAIN) {
        TDP_CUDA_TRY(launch_refine_plain(d_tri, d_tri, d_items, (int)pair_num, d_out, s));
    } else {
        TDP_CUDA_TRY(launch_refine_tuned(d_tri, d_tri, d_items, (int)pair_num, d_out, ctx->d_counter, ctx->d_stats,
                                         ctx->num_sms, ctx->tuned_cfg, s));
    }
    TDP_CUDA_TRY(cudaEventRecord(ctx->ev[1], s));
    std::vector<float4> res(pair_num);
    unsigned long long full = 0;
    TDP_CUDA_TRY(cudaMemcpyAsync(res.data(), d_out, pair_num * sizeof(float4), cudaMemcpyDeviceToHost, s));
    TDP_CUDA_TRY(cudaMemcpyAsync(&full, ctx->d_stats, sizeof(full), cudaMemcpyDeviceToHost, s));
    TDP_CUDA_TRY(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->stats = LastStats();
    ctx->stats.refine_ms = ms;
    ctx->stats.total_ms = ms;
    ctx->stats.tri_pairs = tri_pairs;
    ctx->stats.full_evals = form == TDP_FORM_PLAIN ? (unsigned long long)tri_pairs : full;
    ctx->stats.refine_items = pair_num;
    ctx->stats.refine_launches = 1;
    ctx->stats.kernel_launches = 2;
    for (uint32_t i = 0; i < pair_num; ++i) {
        out[3 * i] = res[i].x;
        out[3 * i + 1] = hausdorff ? res[i].y : FLT_MAX;
        out[3 * i + 2] = hausdorff ? res[i].z : FLT_MAX;
    }
    return TDP_OK;
}

}  // extern "C"
