// bounds_raw.cpp -- tdp_raw_compute_bounds: RAW tile bytes in, the same bytes
// with GPU-computed per-triangle and object-level bounds out.
//
// The tile is made resident (tdp_tile_upload), its bounds are recomputed on the
// device (tdp_tile_compute_bounds, csrc/bounds_kernels.cu), the (proxy,
// hausdorff) pairs are gathered per LOD and copied back, and each voxel's
// block of pairs is written where the RAW format keeps it: right after the
// voxel's 9 floats per triangle at the voxel's (offset, count) of that LOD
// (reference src/storage/tile_IO.cpp:79-172, read back by
// src/spatial/himesh_wrapper.cpp:48-83); the object-level (hausdorff, proxy)
// pairs follow the voxel count after the data block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../csrc/bounds_kernels.cuh"
#include "../../csrc/ctx.cuh"
#include "storage/dev_tile.h"
#include "tdp.h"

using namespace tdp;

namespace {

template <typename Fn>
void parallel_ranges(long n, Fn fn) {
    const long nt = std::max(1L, std::min<long>((long)std::thread::hardware_concurrency(), (n + 4095) / 4096));
    if (nt == 1) { fn(0L, n); return; }
    std::vector<std::thread> pool;
    for (long k = 0; k < nt; ++k) pool.emplace_back([&, k] { fn(n * k / nt, n * (k + 1) / nt); });
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" int tdp_raw_compute_bounds(tdp_ctx* ctx, const void* raw, size_t len, void* out, tdp_bounds_info* info) {
    if (!ctx || !raw || !out) return TDP_ERR_ARG;
    tdp_tile* T = nullptr;
    int rc = tdp_tile_upload(ctx, raw, len, 0, &T);
    if (rc != TDP_OK) return rc;
    struct Release {
        tdp_ctx* c;
        tdp_tile* t;
        ~Release() { tdp_tile_free(c, t); }
    } release{ctx, T};
    if ((rc = tdp_tile_compute_bounds(ctx, T, info))) return rc;
    const TileHost& H = T->host;
    // the (proxy, hausdorff) pairs of every LOD, in the tile's voxel order
    std::vector<float> hd[kNumLods];
    void* dbuf = nullptr;
    size_t most = 0;
    for (int l = 0; l < kNumLods; ++l) most = std::max<size_t>(most, H.n_tris[l]);
    if (most) {
        if (dmalloc(ctx, &dbuf, most * 2 * sizeof(float)) != cudaSuccess)
            return fail(ctx, TDP_ERR_NOMEM, "bound preparation: cannot allocate the gather buffer");
        for (int l = 0; l < kNumLods; ++l) {
            hd[l].resize(2 * (size_t)H.n_tris[l]);
            if (!H.n_tris[l]) continue;
            cudaError_t e = launch_gather_bounds(T->tri[l], H.n_tris[l], (float*)dbuf, ctx->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(hd[l].data(), dbuf, hd[l].size() * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) {
                dfree(ctx, dbuf);
                return fail(ctx, TDP_ERR_CUDA, std::string("bound preparation: ") + cudaGetErrorString(e));
            }
        }
        dfree(ctx, dbuf);
    }
    uint8_t* o = (uint8_t*)out;
    const uint8_t* in = (const uint8_t*)raw;
    if (o != in) {
        parallel_ranges((long)((len + 4095) / 4096), [&](long b, long e) {
            const size_t lo = (size_t)b * 4096, hi = std::min(len, (size_t)e * 4096);
            if (lo < hi) std::memcpy(o + lo, in + lo, hi - lo);
        });
    }
    parallel_ranges(H.n_vox, [&](long b, long e) {
        for (long v = b; v < e; ++v)
            for (int l = 0; l < kNumLods; ++l) {
                const uint32_t n = H.vox_cnt[l][v];
                if (n) std::memcpy(o + H.vox_byte_off[l][v] + 36 * (size_t)n, &hd[l][2 * (size_t)T->h_vtri[l][v]], 8 * (size_t)n);
            }
    });
    for (long k = 0; k < H.n_obj; ++k) {
        uint8_t* p = o + H.obj_data_off[k] + H.obj_data_size[k] + sizeof(uint64_t);
        for (int l = 0; l < kNumLods; ++l) {
            std::memcpy(p + 8 * l, &H.obj_hd[(size_t)k * kNumLods + l], 4);
            std::memcpy(p + 8 * l + 4, &H.obj_phd[(size_t)k * kNumLods + l], 4);
        }
    }
    return TDP_OK;
}
