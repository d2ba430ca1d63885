// tile.cu -- upload of a RAW .dt tile into HBM (tdp_tile_upload / tdp_tile_free).
//
// Replaces Tile::load + HiMesh_Wrapper(RAW) + HiMesh_Wrapper::decode_to and the
// per-chunk packing of triangles into pinned buffers (reference
// src/storage/tile_IO.cpp:13-49, src/spatial/himesh_wrapper.cpp:17-83 and
// :137-169, src/join/SpatialJoin.cpp:169-248): the whole tile, every LOD, is
// made resident once, so no LOD step ever re-packs or re-copies triangles.
//
// The raw bytes are copied to the device in chunks of whole objects and
// unpacked by a kernel (one warp per voxel/LOD segment) into 48-byte triangle
// records.  Every field of a RAW object is 4 or 8 bytes, so every float sits a
// multiple of 4 bytes after its object's first byte; a chunk is copied starting
// at an object's first byte into a 256-byte aligned staging buffer, which makes
// every float 4-byte aligned on the device (checked on the host per segment).
#include <algorithm>
#include <thread>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "attach_kernels.cuh"
#include "ctx.cuh"
#include "storage/dev_tile.h"
#include "storage/host_pool.h"
#include "tile_kernels.cuh"

namespace tdp {

struct TriPtrs {
    float4* p[kNumLods];
};

__global__ void unpack_kernel(const uint8_t* __restrict__ raw, const UnpackSeg* __restrict__ segs, int nseg,
                              TriPtrs tri) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nseg; s += warps) {
        const UnpackSeg g = segs[s];
        const uint32_t n = g.cnt_lod & 0xffffffu;
        float4* dst = tri.p[g.cnt_lod >> 24] + (size_t)g.dst * 3;
        const float* t = reinterpret_cast<const float*>(raw + g.src);
        const float* h = t + 9 * (size_t)n;
        for (uint32_t i = lane; i < n; i += 32) {
            const float* q = t + 9 * (size_t)i;
            dst[3 * (size_t)i + 0] = make_float4(q[0], q[1], q[2], h[2 * i]);
            dst[3 * (size_t)i + 1] = make_float4(q[3], q[4], q[5], h[2 * i + 1]);
            dst[3 * (size_t)i + 2] = make_float4(q[6], q[7], q[8], 0.f);
        }
    }
}

cudaError_t launch_unpack(const uint8_t* raw, const UnpackSeg* segs, int nseg, float4* const* tri, int num_sms,
                          cudaStream_t s) {
    if (nseg <= 0) return cudaSuccess;
    TriPtrs tp;
    for (int l = 0; l < kNumLods; ++l) tp.p[l] = tri[l];
    const int blocks = (int)std::min<size_t>(((size_t)nseg + 7) / 8, (size_t)num_sms * 16);
    unpack_kernel<<<blocks, 256, 0, s>>>(raw, segs, nseg, tp);
    return cudaGetLastError();
}

// fn(b, e) over [0, n) on the host pool's threads (one range for small n)
template <typename Fn>
static void host_parallel(long n, Fn fn) {
    host_ranges(n, 4096, fn);
}

// Device arrays go back to the context's block cache: every caller has
// synchronised the context's stream, or queued the arrays' pending work on it.
void tile_release(tdp_ctx* ctx, tdp_tile* t) {
    if (!t) return;
    block_release(ctx, t->vox);
    block_release(ctx, t->obj_vox);
    block_release(ctx, t->obj_hd);
    block_release(ctx, t->obj_phd);
    for (int l = 0; l < kNumLods; ++l) {
        block_release(ctx, t->tri[l]);  // kept for the next tile of the size
        block_release(ctx, t->vtri[l]);
    }
    block_release(ctx, (void*)t->lazy_data_off);
    block_release(ctx, t->lazy_state);
    block_release(ctx, t->lazy_bytes);
    block_release(ctx, t->d_boxes);
    block_release(ctx, t->box_grid.start);
    block_release(ctx, t->box_grid.items);
    block_release(ctx, t->point_grid.start);
    block_release(ctx, t->point_grid.items);
    delete t;
}

constexpr int kUseHostParse = -1000;

// The attach path with the voxel tables read on the GPU.  Returns TDP_OK (T
// attached) or, with T released in both cases, kUseHostParse (parse on the
// host instead) or an error.
template <typename GrowStage>
static int attach_on_gpu(tdp_ctx* ctx, tdp_tile* T, const uint8_t* buf, const uint8_t* dev_view, size_t len,
                         long max_objects, int slot, GrowStage& grow_stage, std::chrono::steady_clock::time_point t0) {
    auto ms_since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    // A tile of equal-size records (instances of one mesh) needs no walk:
    // the records are placed at the first record's stride when the length is
    // a whole number of strides, and the GPU checks every object's size
    // fields against the first one's (any difference: the host walks it).
    HostVec<RawRec> recs;
    RawRec r0{};
    uint64_t stride = 0;
    const bool strided = max_objects <= 0 && raw_first_record(buf, len, r0, stride) && (len - 1) % stride == 0 &&
                         (len - 1) / stride >= 1024;
    if (!strided && (!walk_raw_dt(buf, len, max_objects, recs) || recs.empty())) {
        tile_release(ctx, T);
        return kUseHostParse;
    }
    const long n = strided ? (long)((len - 1) / stride) : (long)recs.size();
    // voxel counts per chunk of objects, in parallel, then their prefix
    const long nch = std::max(1L, std::min<long>((long)host_threads(), n / 4096));
    std::vector<uint64_t> ch_vox(nch + 1, 0);
    if (strided) {
        for (long k = 0; k < nch; ++k) ch_vox[k + 1] = (uint64_t)(n * (k + 1) / nch) * r0.vnum;
    } else {
        host_for(nch, [&](long k) {
            uint64_t sv = 0;
            for (long o = n * k / nch; o < n * (k + 1) / nch; ++o) sv += recs[o].vnum;
            ch_vox[k + 1] = sv;
        });
        for (long k = 0; k < nch; ++k) ch_vox[k + 1] += ch_vox[k];
    }
    const uint64_t nvox = ch_vox[nch];
    const uint64_t meta_bytes = (uint64_t)n * (2 * kNumLods * 4 + 12) + nvox * 116;
    if (nvox >= 0xffffffffull) {
        tile_release(ctx, T);
        return kUseHostParse;
    }
    TileHost& H = T->host;
    H.n_obj = n;
    H.n_vox = (long)nvox;
    H.obj_vox_off.resize(n + 1);
    H.obj_data_off.resize(n);
    H.obj_data_size.resize(n);
    // the object records go up through the staging slot, obj_vox[n] after them
    grow_stage(std::max((size_t)(n + 1) * sizeof(AttachRec), (size_t)9 * n * sizeof(float)) + 64);
    AttachRec* ar = (AttachRec*)ctx->hstage[slot];
    std::vector<AttachRec> ar_pageable;
    if (!ar) {
        ar_pageable.resize(n + 1);
        ar = ar_pageable.data();
    }
    // strided: the GPU places the records itself (k_parse_tables), so only
    // the host's copies of the object arrays are written here
    host_for(nch, [&](long k) {
        uint32_t v0 = (uint32_t)ch_vox[k];
        for (long o = n * k / nch; o < n * (k + 1) / nch; ++o) {
            const RawRec r = strided ? RawRec{r0.data_off + o * stride, r0.data_size, r0.meta + o * stride, r0.vnum}
                                     : recs[o];
            if (!strided) ar[o] = AttachRec{r.data_off, r.data_size, r.meta, (uint32_t)r.vnum, v0};
            H.obj_vox_off[o] = v0;
            H.obj_data_off[o] = r.data_off;
            H.obj_data_size[o] = r.data_size;
            v0 += (uint32_t)r.vnum;
        }
    });
    const uint32_t v0 = (uint32_t)nvox;
    H.obj_vox_off[n] = v0;
    uint32_t* nvox_src = reinterpret_cast<uint32_t*>(ar + n);
    *nvox_src = v0;
    T->parse_ms = ms_since(t0);
    const auto ta = std::chrono::steady_clock::now();
    T->n_obj = n;
    T->n_vox = (long)nvox;
    cudaStream_t s = ctx->stream;
    auto alloc = [&](void** p, size_t bytes) -> int {
        if (block_alloc(ctx, p, bytes) != cudaSuccess)
            return fail(ctx, TDP_ERR_NOMEM, "tile attach: cannot allocate " + std::to_string(bytes) + " bytes" +
                                                (ctx->budget ? " within the context budget" : ""));
        T->device_bytes += bytes;
        return TDP_OK;
    };
#define GTRY(x) do { int _r = (x); if (_r) { cudaStreamSynchronize(s); tile_release(ctx, T); return _r; } } while (0)
#define GCTRY(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { cudaStreamSynchronize(s); tile_release(ctx, T); return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } } while (0)
    GTRY(alloc((void**)&T->vox, (size_t)nvox * 3 * sizeof(float4)));
    GTRY(alloc((void**)&T->obj_vox, (size_t)(n + 1) * sizeof(uint32_t)));
    GTRY(alloc((void**)&T->obj_hd, (size_t)n * kNumLods * sizeof(float)));
    GTRY(alloc((void**)&T->obj_phd, (size_t)n * kNumLods * sizeof(float)));
    for (int l = 0; l < kNumLods; ++l) GTRY(alloc((void**)&T->vtri[l], (size_t)(nvox + 1) * sizeof(uint32_t)));
    GTRY(alloc((void**)&T->lazy_data_off, (size_t)n * sizeof(uint64_t)));
    GTRY(alloc((void**)&T->lazy_state, (size_t)kNumLods * std::max<uint64_t>(nvox, 1) * sizeof(unsigned)));
    GTRY(alloc((void**)&T->lazy_bytes, sizeof(unsigned long long)));
    GTRY(alloc((void**)&T->d_boxes, (size_t)n * 9 * sizeof(float)));
    T->boxes_n = n;
    Buf& recs_d = ctx->scratch[96];
    Buf& off4 = ctx->scratch[97];
    Buf& vobj = ctx->scratch[98];
    Buf& tmp = ctx->scratch[99];
    Buf& ctr = ctx->scratch[100];
    GTRY(ensure(ctx, recs_d, (size_t)(n + 1) * sizeof(AttachRec)));
    GTRY(ensure(ctx, off4, (size_t)kNumLods * std::max<uint64_t>(nvox, 1) * sizeof(uint32_t)));
    GTRY(ensure(ctx, vobj, (size_t)std::max<uint64_t>(nvox, 1) * sizeof(uint32_t)));
    GTRY(ensure(ctx, ctr, 16 * sizeof(unsigned long long)));
    AttachOut o{};
    o.vox = T->vox;
    o.obj_vox = T->obj_vox;
    o.obj_hd = T->obj_hd;
    o.obj_phd = T->obj_phd;
    o.boxes = T->d_boxes;
    o.data_off = T->lazy_data_off;
    for (int l = 0; l < kNumLods; ++l) {
        o.vtri[l] = T->vtri[l];
        o.off4[l] = (uint32_t*)off4.p + (size_t)l * nvox;
    }
    o.vobj = (uint32_t*)vobj.p;
    o.n_tris = (unsigned long long*)ctr.p;
    o.first_bad = (unsigned long long*)ctr.p + 8;
    size_t scan_bytes = 0;
    GCTRY(launch_attach_tables(dev_view, nullptr, n, (long)nvox, o, nullptr, scan_bytes, ctx->num_sms, s));
    GTRY(ensure(ctx, tmp, scan_bytes + 16));
    T->alloc_ms = ms_since(ta);
    const auto tm = std::chrono::steady_clock::now();
    if (!strided) GCTRY(cudaMemcpyAsync(recs_d.p, ar, (size_t)n * sizeof(AttachRec), cudaMemcpyHostToDevice, s));
    GCTRY(cudaMemcpyAsync(T->obj_vox + n, nvox_src, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    GCTRY(cudaMemsetAsync(ctr.p, 0, 8 * sizeof(unsigned long long), s));
    GCTRY(cudaMemsetAsync((unsigned long long*)ctr.p + 8, 0xff, sizeof(unsigned long long), s));
    AttachStride ast{};
    if (strided) ast = AttachStride{1, stride, AttachRec{r0.data_off, r0.data_size, r0.meta, (uint32_t)r0.vnum, 0u}};
    GCTRY(launch_attach_tables(dev_view, (const AttachRec*)recs_d.p, n, (long)nvox, o, tmp.p, scan_bytes,
                               ctx->num_sms, s, ast));
    unsigned long long res[9] = {0};
    GCTRY(cudaMemcpyAsync(res, ctr.p, 9 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    // the object boxes and transforms come back through the staging slot (its
    // records have gone up by then, in stream order) and are spread into the
    // host arrays after the synchronisation
    H.obj_box.resize((size_t)6 * n);
    H.obj_xf.resize((size_t)3 * n);
    float* box_stage = ar_pageable.empty() ? reinterpret_cast<float*>(ctx->hstage[slot]) : nullptr;
    GCTRY(cudaMemcpyAsync(box_stage ? box_stage : H.obj_box.data(), T->d_boxes,
                          (size_t)(box_stage ? 9 : 6) * n * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (!box_stage)
        GCTRY(cudaMemcpyAsync(H.obj_xf.data(), T->d_boxes + 6 * n, (size_t)3 * n * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
    if (!ctx->hstage_ev[slot]) GCTRY(cudaEventCreateWithFlags(&ctx->hstage_ev[slot], cudaEventDisableTiming));
    GCTRY(cudaEventRecord(ctx->hstage_ev[slot], s));
    GCTRY(cudaStreamSynchronize(s));
    if (box_stage)
        host_ranges(9 * n, 1 << 16, [&](long b, long e) {
            const long m = std::min(e, 6 * n);
            if (b < m) std::memcpy(H.obj_box.data() + b, box_stage + b, (size_t)(m - b) * sizeof(float));
            if (e > 6 * n) {
                const long xb = std::max(b, 6 * n);
                std::memcpy(H.obj_xf.data() + (xb - 6 * n), box_stage + xb, (size_t)(e - xb) * sizeof(float));
            }
        });
    if (res[8] != ~0ull) {  // a check failed: the host parser reports it
        tile_release(ctx, T);
        return kUseHostParse;
    }
    for (int l = 0; l < kNumLods; ++l) {
        if (res[l] >= 0xffffffffull) {
            tile_release(ctx, T);
            return fail(ctx, TDP_ERR_FORMAT, "more than 2^32 triangles in one LOD");
        }
        H.n_tris[l] = res[l];
    }
    for (int l = 0; l < kNumLods; ++l) GTRY(alloc((void**)&T->tri[l], (size_t)H.n_tris[l] * 3 * sizeof(float4)));
    GCTRY(cudaMemsetAsync(T->lazy_state, 0, (size_t)kNumLods * nvox * sizeof(unsigned), s));
    GCTRY(cudaMemsetAsync(T->lazy_bytes, 0, sizeof(unsigned long long), s));
    if (ctx->flags & TDP_CTX_POISON)
        for (int l = 0; l < kNumLods; ++l)
            GCTRY(cudaMemsetAsync(T->tri[l], 0xff, (size_t)H.n_tris[l] * 3 * sizeof(float4), s));
#undef GTRY
#undef GCTRY
    T->h2d_bytes = (size_t)n * sizeof(AttachRec) + meta_bytes;  // the records, and the tables the GPU read
    T->meta_ms = ms_since(tm);
    T->lazy_raw = dev_view;
    T->lazy_on = true;
    T->lazy_stride = (long)nvox;
    T->load_ms = ms_since(t0);
    return TDP_OK;
}

// Parse, validate and make a tile resident (attach == false), or attach it:
// voxel and object metadata resident, triangle records allocated but filled
// by the joins that need them, straight from the page-locked host bytes.
int tile_load(tdp_ctx* ctx, const void* raw_dt, size_t len, long max_objects, bool attach, tdp_tile** out) {
    if (!ctx || !out) return TDP_ERR_ARG;
    *out = nullptr;
    if (!raw_dt) return fail(ctx, TDP_ERR_ARG, "null tile buffer");
    cudaSetDevice(ctx->device);
    const uint8_t* buf = (const uint8_t*)raw_dt;
    const uint8_t* dev_view = nullptr;
    if (attach) {
        // the bytes must be page-locked (cudaHostRegister / cudaHostAlloc), so
        // that kernels can read them, from the first byte to the last
        cudaPointerAttributes a0{}, a1{};
        void* dp = nullptr;
        if (len == 0 || cudaPointerGetAttributes(&a0, buf) != cudaSuccess || a0.type != cudaMemoryTypeHost ||
            cudaPointerGetAttributes(&a1, buf + len - 1) != cudaSuccess || a1.type != cudaMemoryTypeHost ||
            cudaHostGetDevicePointer(&dp, (void*)buf, 0) != cudaSuccess || !dp) {
            cudaGetLastError();
            return fail(ctx, TDP_ERR_ARG, "tdp_tile_attach needs page-locked host memory (cudaHostRegister or "
                                          "cudaHostAlloc) covering the whole tile; use tdp_tile_upload otherwise");
        }
        dev_view = (const uint8_t*)dp;
    }
    tdp_tile* T = new tdp_tile();
    T->device = ctx->device;
    std::string err;
    const auto t0 = std::chrono::steady_clock::now();
    auto ms_since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    // The metadata go up through one of the context's two page-locked staging
    // buffers, laid out [voxel records][data-block offsets][vtri x 5]
    // [obj_vox][obj_hd][obj_phd]; the parser writes the voxel records into it
    // directly.  The buffer is written only once its previous copies are done.
    const int slot = ctx->hstage_next;
    ctx->hstage_next ^= 1;
    auto wait_slot = [&] {
        if (ctx->hstage_ev[slot]) cudaEventSynchronize(ctx->hstage_ev[slot]);
    };
    auto stage_bytes = [attach](long n_vox, long n_obj) {
        return (size_t)n_vox * 3 * sizeof(float4) + (attach ? (size_t)n_obj * sizeof(uint64_t) : 0) +
               kNumLods * (size_t)(n_vox + 1) * sizeof(uint32_t) + (size_t)(n_obj + 1) * sizeof(uint32_t) +
               2 * (size_t)n_obj * kNumLods * sizeof(float) + 64;
    };
    auto grow_stage = [&](size_t need) {
        wait_slot();
        if (need <= ctx->hstage_cap[slot]) return;
        if (ctx->hstage[slot]) cudaFreeHost(ctx->hstage[slot]);
        ctx->hstage[slot] = nullptr;
        ctx->hstage_cap[slot] = 0;
        if (cudaHostAlloc(&ctx->hstage[slot], need + need / 4, cudaHostAllocDefault) == cudaSuccess)
            ctx->hstage_cap[slot] = need + need / 4;
        else { cudaGetLastError(); ctx->hstage[slot] = nullptr; }
    };
    // ---- attach: the host walks the size fields, the GPU reads the voxel tables ----
    // (csrc/attach_kernels.cu).  A tile the walk cannot take, or whose tables
    // fail a check, goes through the host parser below, which reports the
    // first error in file order.
    if (attach) {
        const int grc = attach_on_gpu(ctx, T, buf, dev_view, len, max_objects, slot, grow_stage, t0);
        if (grc == TDP_OK) {
            *out = T;
            return TDP_OK;
        }
        if (grc != kUseHostParse) return grc;  // T released
        T = new tdp_tile();
        T->device = ctx->device;
    }
    int rc = parse_raw_dt(buf, len, max_objects, T->host, err, [&](long n_vox, long n_obj) -> float* {
        grow_stage(stage_bytes(n_vox, n_obj));
        return (float*)ctx->hstage[slot];  // nullptr when page-locked memory is short
    });
    T->parse_ms = ms_since(t0);
    if (rc != TDP_OK) {
        delete T;
        return fail(ctx, rc, err);
    }
    TileHost& H = T->host;
    T->n_obj = H.n_obj;
    T->n_vox = H.n_vox;
    for (int l = 0; l < kNumLods; ++l)
        if (H.n_tris[l] >= 0xffffffffull) { delete T; return fail(ctx, TDP_ERR_FORMAT, "more than 2^32 triangles in one LOD"); }
    if (attach && H.first_noncanonical >= 0) {
        // fetches locate a voxel's bytes from the prefix arrays, which needs
        // the layout the reference's writer produces (checked by the parser)
        const long o = H.first_noncanonical;
        delete T;
        return fail(ctx, TDP_ERR_FORMAT, "object " + std::to_string(o) +
                                             " does not keep its voxels' triangles in LOD and voxel "
                                             "order; use tdp_tile_upload for this tile");
    }
    const auto ta = std::chrono::steady_clock::now();
    auto alloc = [&](void** p, size_t bytes) -> int {
        if (block_alloc(ctx, p, bytes) != cudaSuccess)
            return fail(ctx, TDP_ERR_NOMEM, "tile upload: cannot allocate " + std::to_string(bytes) + " bytes" +
                                                (ctx->budget ? " within the context budget" : ""));
        T->device_bytes += bytes;
        return TDP_OK;
    };
    cudaStream_t s = ctx->stream;
    // CTRY synchronises the stream before it returns an error: copies already
    // queued from the staging slot have finished by then, so the slot's event
    // (recorded only on success) cannot let a later attach rewrite page-locked
    // memory that a queued copy still reads.
#define TRY(x) do { int _r = (x); if (_r) { tile_release(ctx, T); return _r; } } while (0)
#define CTRY(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { cudaStreamSynchronize(s); tile_release(ctx, T); return fail(ctx, TDP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); } } while (0)
    TRY(alloc((void**)&T->vox, (size_t)H.n_vox * 3 * sizeof(float4)));
    TRY(alloc((void**)&T->obj_vox, (size_t)(H.n_obj + 1) * sizeof(uint32_t)));
    TRY(alloc((void**)&T->obj_hd, (size_t)H.n_obj * kNumLods * sizeof(float)));
    TRY(alloc((void**)&T->obj_phd, (size_t)H.n_obj * kNumLods * sizeof(float)));
    for (int l = 0; l < kNumLods; ++l) {
        TRY(alloc((void**)&T->tri[l], (size_t)H.n_tris[l] * 3 * sizeof(float4)));
        TRY(alloc((void**)&T->vtri[l], (size_t)(H.n_vox + 1) * sizeof(uint32_t)));
    }
    if (attach) {
        TRY(alloc((void**)&T->lazy_data_off, (size_t)std::max<long>(H.n_obj, 1) * sizeof(uint64_t)));
        TRY(alloc((void**)&T->lazy_state, (size_t)kNumLods * std::max<long>(H.n_vox, 1) * sizeof(unsigned)));
        TRY(alloc((void**)&T->lazy_bytes, sizeof(unsigned long long)));
    }
    T->alloc_ms = ms_since(ta);
    const auto tm = std::chrono::steady_clock::now();
    {
        // The voxel records (staged by the parser) start their copy, then
        // host threads write the prefix of triangle counts per LOD into the
        // tile's host copy and the staging slot at once.
        const size_t v4_bytes = (size_t)H.n_vox * 3 * sizeof(float4);
        const size_t do_bytes = attach ? (size_t)H.n_obj * sizeof(uint64_t) : 0;
        const size_t vt_bytes = (size_t)(H.n_vox + 1) * sizeof(uint32_t);
        const size_t ov_bytes = H.obj_vox_off.size() * 4, hd_bytes = H.obj_hd.size() * 4;
        const bool staged = H.vox_box.empty();  // the parser wrote the voxel records into the staging buffer
        if (!staged) grow_stage(stage_bytes(H.n_vox, H.n_obj));
        uint8_t* stg = (uint8_t*)ctx->hstage[slot];  // nullptr: copy from pageable memory
        uint32_t* vt_stage[kNumLods] = {};
        uint32_t* vt_host[kNumLods] = {};
        for (int l = 0; l < kNumLods; ++l) {
            T->h_vtri[l].resize(H.n_vox + 1);
            vt_host[l] = T->h_vtri[l].data();
            if (stg) vt_stage[l] = (uint32_t*)(stg + v4_bytes + do_bytes + l * vt_bytes);
        }
        std::vector<float4> v4_pageable;
        float4* v4 = nullptr;
        if (stg) v4 = (float4*)stg;
        else { v4_pageable.resize((size_t)H.n_vox * 3); v4 = v4_pageable.data(); }
        if (!staged)
            host_parallel(H.n_vox, [&](long b, long e) {
                for (long v = b; v < e; ++v) {
                    const float* x = &H.vox_box[9 * v];
                    v4[3 * v + 0] = make_float4(x[0], x[1], x[2], 0.f);
                    v4[3 * v + 1] = make_float4(x[3], x[4], x[5], 0.f);
                    v4[3 * v + 2] = make_float4(x[6], x[7], x[8], 0.f);
                }
            });
        const void* src_do = H.obj_data_off.data();
        if (stg && attach) {
            std::memcpy(stg + v4_bytes, src_do, do_bytes);
            src_do = stg + v4_bytes;
        }
        CTRY(cudaMemcpyAsync(T->vox, v4, v4_bytes, cudaMemcpyHostToDevice, s));
        if (attach) CTRY(cudaMemcpyAsync(T->lazy_data_off, src_do, do_bytes, cudaMemcpyHostToDevice, s));
        vtri_prefix(H, vt_host, vt_stage);
        const void* src_vt[kNumLods];
        const void* src_ov = H.obj_vox_off.data();
        const void* src_hd = H.obj_hd.data();
        const void* src_phd = H.obj_phd.data();
        if (stg) {
            uint8_t* p = stg + v4_bytes + do_bytes + kNumLods * vt_bytes;
            for (int l = 0; l < kNumLods; ++l) src_vt[l] = vt_stage[l];
            std::memcpy(p, src_ov, ov_bytes); src_ov = p; p += ov_bytes;
            std::memcpy(p, src_hd, hd_bytes); src_hd = p; p += hd_bytes;
            std::memcpy(p, src_phd, hd_bytes); src_phd = p;
        } else {
            for (int l = 0; l < kNumLods; ++l) src_vt[l] = T->h_vtri[l].data();
        }
        for (int l = 0; l < kNumLods; ++l)
            CTRY(cudaMemcpyAsync(T->vtri[l], src_vt[l], vt_bytes, cudaMemcpyHostToDevice, s));
        CTRY(cudaMemcpyAsync(T->obj_vox, src_ov, ov_bytes, cudaMemcpyHostToDevice, s));
        CTRY(cudaMemcpyAsync(T->obj_hd, src_hd, hd_bytes, cudaMemcpyHostToDevice, s));
        CTRY(cudaMemcpyAsync(T->obj_phd, src_phd, hd_bytes, cudaMemcpyHostToDevice, s));
        T->h2d_bytes += v4_bytes + do_bytes + ov_bytes + 2 * hd_bytes + kNumLods * vt_bytes;
        if (attach) {
            CTRY(cudaMemsetAsync(T->lazy_state, 0, (size_t)kNumLods * H.n_vox * sizeof(unsigned), s));
            CTRY(cudaMemsetAsync(T->lazy_bytes, 0, sizeof(unsigned long long), s));
            if (ctx->flags & TDP_CTX_POISON)
                for (int l = 0; l < kNumLods; ++l)
                    CTRY(cudaMemsetAsync(T->tri[l], 0xff, (size_t)H.n_tris[l] * 3 * sizeof(float4), s));
        }
        // An attach returns with its copies queued: every later use of the
        // tile is ordered after them on the context's stream, and the event
        // keeps this staging buffer from being rewritten before they finish.
        if (!ctx->hstage_ev[slot]) CTRY(cudaEventCreateWithFlags(&ctx->hstage_ev[slot], cudaEventDisableTiming));
        CTRY(cudaEventRecord(ctx->hstage_ev[slot], s));
        if (!attach || !stg) CTRY(cudaStreamSynchronize(s));
    }
    T->meta_ms = ms_since(tm);
    if (attach) {
        T->lazy_raw = dev_view;
        T->lazy_on = true;
        T->lazy_stride = H.n_vox;
        T->load_ms = ms_since(t0);
        *out = T;
        return TDP_OK;
    }
    // chunked copy + unpack of the triangle data, whole objects per chunk
    const size_t kChunk = (size_t)1 << 30;
    Buf& stage = ctx->scratch[12];
    Buf& segbuf = ctx->scratch[13];
    TriPtrs tp;
    for (int l = 0; l < kNumLods; ++l) tp.p[l] = T->tri[l];
    std::vector<UnpackSeg> segs;
    long o0 = 0;
    while (o0 < H.n_obj) {
        // the object's first byte: its floats sit at a multiple of 4 bytes from it
        const uint64_t base = H.obj_data_off[o0] - 8;
        long o1 = o0 + 1;
        while (o1 < H.n_obj && H.obj_data_off[o1] + H.obj_data_size[o1] - base <= kChunk) ++o1;
        const uint64_t end = H.obj_data_off[o1 - 1] + H.obj_data_size[o1 - 1];
        const size_t bytes = (size_t)(end - base);
        TRY(ensure(ctx, stage, bytes + 16));
        segs.clear();
        for (long o = o0; o < o1; ++o)
            for (uint32_t v = H.obj_vox_off[o]; v < H.obj_vox_off[o + 1]; ++v)
                for (int l = 0; l < kNumLods; ++l) {
                    uint32_t n = H.vox_cnt[l][v];
                    if (!n) continue;
                    const uint64_t src = H.vox_byte_off[l][v] - base;
                    if ((src & 3u) || src + (uint64_t)n * 44 > bytes) {  // never launch a misaligned read
                        tile_release(ctx, T);
                        return fail(ctx, TDP_ERR_FORMAT, "triangle block of object " + std::to_string(o) +
                                                             " is not 4-byte aligned within its object");
                    }
                    segs.push_back({src, T->h_vtri[l][v], n | ((uint32_t)l << 24)});
                }
        TRY(ensure(ctx, segbuf, std::max<size_t>(segs.size(), 1) * sizeof(UnpackSeg)));
        CTRY(cudaMemcpyAsync(stage.p, buf + base, bytes, cudaMemcpyHostToDevice, s));
        T->h2d_bytes += bytes + segs.size() * sizeof(UnpackSeg);
        CTRY(cudaMemcpyAsync(segbuf.p, segs.data(), segs.size() * sizeof(UnpackSeg), cudaMemcpyHostToDevice, s));
        if (!segs.empty()) {
            int blocks = (int)std::min<size_t>((segs.size() + 7) / 8, (size_t)ctx->num_sms * 16);
            unpack_kernel<<<blocks, 256, 0, s>>>((const uint8_t*)stage.p, (const UnpackSeg*)segbuf.p, (int)segs.size(), tp);
            CTRY(cudaGetLastError());
        }
        CTRY(cudaStreamSynchronize(s));
        o0 = o1;
    }
#undef TRY
#undef CTRY
    T->load_ms = ms_since(t0);
    *out = T;
    return TDP_OK;
}

}  // namespace tdp

using namespace tdp;

extern "C" {

int tdp_tile_upload(tdp_ctx* ctx, const void* raw_dt, size_t len, long max_objects, tdp_tile** out) {
    return tile_load(ctx, raw_dt, len, max_objects, false, out);
}

int tdp_tile_attach(tdp_ctx* ctx, const void* raw_dt, size_t len, long max_objects, tdp_tile** out) {
    return tile_load(ctx, raw_dt, len, max_objects, true, out);
}

int tdp_host_alloc(size_t bytes, void** out) {
    if (!out) return TDP_ERR_ARG;
    *out = nullptr;
    if (bytes == 0) return TDP_ERR_ARG;
    if (cudaHostAlloc(out, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return TDP_ERR_NOMEM;
    }
    return TDP_OK;
}

int tdp_host_free(void* p) {
    if (!p) return TDP_ERR_ARG;
    return cudaFreeHost(p) == cudaSuccess ? TDP_OK : TDP_ERR_CUDA;
}

int tdp_tile_free(tdp_ctx* ctx, tdp_tile* tile) {
    if (!ctx || !tile) return TDP_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    tile_release(ctx, tile);
    return TDP_OK;
}

int tdp_tile_get_info(const tdp_tile* t, tdp_tile_info* o) {
    if (!t || !o) return TDP_ERR_ARG;
    o->n_objects = t->n_obj;
    o->n_voxels = t->n_vox;
    for (int l = 0; l < kNumLods; ++l) o->n_tris[l] = (long)t->host.n_tris[l];
    o->device_bytes = t->device_bytes;
    o->h2d_bytes = t->h2d_bytes;
    o->attached = t->lazy_raw != nullptr;
    o->parse_ms = t->parse_ms;
    o->alloc_ms = t->alloc_ms;
    o->load_ms = t->load_ms;
    o->meta_ms = t->meta_ms;
    return TDP_OK;
}

}  // extern "C"
