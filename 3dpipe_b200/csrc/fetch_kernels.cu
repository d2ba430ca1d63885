// fetch_kernels.cu -- on-demand triangle fetch for attached tiles (see
// fetch_kernels.cuh).
//
// A voxel's bytes at one LOD sit in its object's data block in the RAW layout
// that the reference's writer produces (src/storage/tile_IO.cpp:79-172): for
// each LOD, for each voxel, 9 floats per triangle, then (proxy, hausdorff) per
// triangle.  tdp_tile_attach accepts only tiles in that layout, so the offset
// of (voxel v, LOD l) inside object o's block is 44 bytes times the triangles
// the object holds at the LODs before l plus those of o's voxels before v at
// l -- all read from the tile's resident prefix arrays, nothing extra is
// uploaded.  Every float of a RAW object sits a multiple of 4 bytes after the
// object's first byte, but the objects follow a one-byte header, so the host
// floats are read as aligned 32-bit words and realigned with a funnel shift
// (the word after the last float still lies inside the object's record: the
// voxel table and the transform follow the data block).  A warp moves 32
// triangles at a time: coalesced word reads from host memory into shared
// memory, then one 48-byte record per lane.  Serving arenas use the same
// fetch with absolute addresses: each object's data block lives in its own
// request's page-locked buffer.
#include "fetch_kernels.cuh"

#include <algorithm>

#include "storage/dev_tile.h"

namespace tdp {

namespace {

constexpr int kFetchWarps = 8;
constexpr int kStageWords = 32 * 11 + 1;

// last index i in [0, n) with a[i] <= x (a ascending, a[0] <= x)
__device__ inline long last_le(const uint32_t* a, long n, uint32_t x) {
    long lo = 0, hi = n - 1;
    while (lo < hi) {
        const long mid = (lo + hi + 1) >> 1;
        if (a[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// stage[k] = the float that starts sh/8 bytes into word k of src, k < cnt
// (cnt <= 32 * R - 1): lane j holds words j, j + 32, ...; word k + 1, which
// the realignment needs, is the next lane's (lane 0's next round for lane 31).
// Reads exactly words 0..cnt of src.
template <int R>
__device__ __forceinline__ void copy_words(const uint32_t* src, uint32_t cnt, unsigned sh, int lane,
                                           uint32_t* stage) {
    uint32_t w[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t k = 32 * r + lane;
        w[r] = k <= cnt && (sh || k < cnt) ? src[k] : 0u;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t up = __shfl_down_sync(0xffffffffu, w[r], 1);
        const uint32_t wrap = __shfl_sync(0xffffffffu, r + 1 < R ? w[r + 1 < R ? r + 1 : r] : 0u, 0);
        const uint32_t next = lane < 31 ? up : wrap;
        const uint32_t k = 32 * r + lane;
        if (k < cnt) stage[k] = sh ? __funnelshift_r(w[r], next, sh) : w[r];
    }
}

// copy voxel v's n triangles at LOD index lod (first record off) from the host
// bytes into the tile's records, if this warp is the first to claim the voxel
__device__ void fetch_voxel(const LazyTile& L, int lod, long v, uint32_t off, uint32_t n, uint32_t* stage) {
    const int lane = threadIdx.x & 31;
    unsigned prev = 1;
    if (lane == 0) prev = atomicCAS(L.state + (size_t)lod * L.stride + v, 0u, 1u);
    prev = __shfl_sync(0xffffffffu, prev, 0);
    if (prev != 0u) return;
    const long o = last_le(L.obj_vox, L.n_obj + 1, (uint32_t)v);
    const uint32_t vb = L.obj_vox[o], ve = L.obj_vox[o + 1];
    uint64_t before = off - L.vtri[lod][vb];
    for (int l = 0; l < lod; ++l) before += L.vtri[l][ve] - L.vtri[l][vb];
    const uintptr_t base = reinterpret_cast<uintptr_t>(L.raw) + L.data_off[o] + 44 * before;
    const uint32_t* W = reinterpret_cast<const uint32_t*>(base & ~uintptr_t(3));
    const unsigned sh = (unsigned)(base & 3) * 8;
    float4* dst = L.tri[lod] + 3 * (size_t)off;
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t m = min(32u, n - c0);
        // the 9m triangle words and 2m bound words of these m triangles, plus
        // the word after each run (for the realignment): every load issued
        // before any is used; the next word comes from the next lane
        copy_words<10>(W + 9 * (uint64_t)c0, 9 * m, sh, lane, stage);
        copy_words<3>(W + 9 * (uint64_t)n + 2 * (uint64_t)c0, 2 * m, sh, lane, stage + 9 * m);
        __syncwarp();
        if (lane < m) {
            const float* f = reinterpret_cast<const float*>(stage + 9 * lane);
            const float* h = reinterpret_cast<const float*>(stage + 9 * m + 2 * lane);
            float4* r = dst + 3 * (size_t)(c0 + lane);
            r[0] = make_float4(f[0], f[1], f[2], h[0]);
            r[1] = make_float4(f[3], f[4], f[5], h[1]);
            r[2] = make_float4(f[6], f[7], f[8], 0.f);
        }
        __syncwarp();
    }
    if (lane == 0) atomicAdd(L.bytes, 44ull * n);
}

__global__ void __launch_bounds__(kFetchWarps * 32) k_fetch_items(const RefineItem* __restrict__ items,
                                                                  const unsigned* n_dev, long n_host, int lod,
                                                                  LazyTile A, LazyTile B) {
    __shared__ uint32_t stage[kFetchWarps][kStageWords];
    uint32_t* st = stage[threadIdx.x >> 5];
    const long n = n_dev ? (long)*n_dev : n_host;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const RefineItem it = items[i];
        if (A.on && it.a_cnt) fetch_voxel(A, lod, last_le(A.vtri[lod], A.n_vox + 1, it.a_off), it.a_off, it.a_cnt, st);
        if (B.on && it.b_cnt) fetch_voxel(B, lod, last_le(B.vtri[lod], B.n_vox + 1, it.b_off), it.b_off, it.b_cnt, st);
    }
}

__global__ void __launch_bounds__(kFetchWarps * 32) k_fetch_all(LazyTile L) {
    __shared__ uint32_t stage[kFetchWarps][kStageWords];
    uint32_t* st = stage[threadIdx.x >> 5];
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < kNumLods * L.n_vox; i += warps) {
        const int lod = (int)(i / L.n_vox);
        const long v = i - (long)lod * L.n_vox;
        const uint32_t off = L.vtri[lod][v], n = L.vtri[lod][v + 1] - off;
        if (n) fetch_voxel(L, lod, v, off, n, st);
    }
}

// lanes test 32 voxel pairs at once; the warp then fetches the flagged ones'
// voxels one pair at a time (fetch_voxel is warp-cooperative and claims each
// voxel once, so voxels shared by many pairs cost one state-word read each)
__global__ void __launch_bounds__(kFetchWarps * 32) k_prefetch_pairs(const uint8_t* __restrict__ valive,
                                                                     const int* __restrict__ vpair,
                                                                     const uint8_t* pstat,
                                                                     const int* __restrict__ vpa,
                                                                     const int* __restrict__ vpb, int64_t V, int lod,
                                                                     LazyTile A, LazyTile B) {
    __shared__ uint32_t stage[kFetchWarps][kStageWords];
    uint32_t* st = stage[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < V; base += warps * 32) {
        const int64_t v = base + lane;
        const bool want = v < V && valive[v] && pstat[vpair[v]] == 0;
        unsigned m = __ballot_sync(0xffffffffu, want);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const int64_t u = base + src;
            if (A.on) {
                const long a = vpa[u];
                const uint32_t off = A.vtri[lod][a], n = A.vtri[lod][a + 1] - off;
                if (n) fetch_voxel(A, lod, a, off, n, st);
            }
            if (B.on) {
                const long b = vpb[u];
                const uint32_t off = B.vtri[lod][b], n = B.vtri[lod][b + 1] - off;
                if (n) fetch_voxel(B, lod, b, off, n, st);
            }
        }
    }
}

}  // namespace

cudaError_t launch_prefetch_pairs(const uint8_t* valive, const int* vpair, const uint8_t* pstat, const int* vpa,
                                  const int* vpb, int64_t V, int lod, const LazyTile& a, const LazyTile& b,
                                  int num_sms, cudaStream_t s) {
    if ((!a.on && !b.on) || V <= 0) return cudaSuccess;
    const int64_t blocks_needed = (V + 32 * kFetchWarps - 1) / (32 * kFetchWarps);
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(blocks_needed, (int64_t)num_sms * 8));
    k_prefetch_pairs<<<blocks, kFetchWarps * 32, 0, s>>>(valive, vpair, pstat, vpa, vpb, V, lod, a, b);
    return cudaGetLastError();
}

LazyTile lazy_view(const tdp_tile* t) {
    LazyTile L;
    if (!t || !t->lazy_on) return L;
    L.on = true;
    L.raw = t->lazy_raw;
    L.data_off = t->lazy_data_off;
    L.obj_vox = t->obj_vox;
    for (int l = 0; l < kNumLods; ++l) {
        L.vtri[l] = t->vtri[l];
        L.tri[l] = t->tri[l];
    }
    L.state = t->lazy_state;
    L.stride = t->lazy_stride;
    L.bytes = t->lazy_bytes;
    L.n_vox = t->n_vox;
    L.n_obj = t->n_obj;
    return L;
}

cudaError_t launch_fetch_items(const RefineItem* items, const unsigned* n_dev, long n_host, int lod,
                               const LazyTile& a, const LazyTile& b, int num_sms, cudaStream_t s) {
    if (!a.on && !b.on) return cudaSuccess;
    if (!n_dev && n_host <= 0) return cudaSuccess;
    const long blocks_needed = n_dev ? (long)num_sms * 8 : (n_host + kFetchWarps - 1) / kFetchWarps;
    const int blocks = (int)std::max(1L, std::min<long>(blocks_needed, (long)num_sms * 8));
    k_fetch_items<<<blocks, kFetchWarps * 32, 0, s>>>(items, n_dev, n_host, lod, a, b);
    return cudaGetLastError();
}

cudaError_t launch_fetch_all(const LazyTile& t, int num_sms, cudaStream_t s) {
    if (!t.on || t.n_vox == 0) return cudaSuccess;
    k_fetch_all<<<num_sms * 8, kFetchWarps * 32, 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace tdp
