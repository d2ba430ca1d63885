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
// 16-byte chunks that can hold 9 x 32 triangle words (73 at any alignment)
// and 2 x 32 bound words (17), rounded up
constexpr int kTriChunks = 74;
constexpr int kHdChunks = 18;
constexpr int kStageT = 4 * kTriChunks;         // words
constexpr int kStageWords = kStageT + 4 * kHdChunks;
constexpr unsigned kWanted = 2u;                // state: marked by a mark pass

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

// device-view address of voxel v's first triangle at LOD index lod (first
// record off): its object's data block, then the triangles of the object's
// LODs before lod and of its voxels before v at lod, 44 bytes each
__device__ __forceinline__ uintptr_t voxel_src(const LazyTile& L, int lod, long v, uint32_t off) {
    const long o = last_le(L.obj_vox, L.n_obj + 1, (uint32_t)v);
    const uint32_t vb = L.obj_vox[o], ve = L.obj_vox[o + 1];
    uint64_t before = off - L.vtri[lod][vb];
    for (int l = 0; l < lod; ++l) before += L.vtri[l][ve] - L.vtri[l][vb];
    return reinterpret_cast<uintptr_t>(L.raw) + L.data_off[o] + 44 * before;
}

__device__ __forceinline__ void mark(const LazyTile& L, int lod, long v) {
    unsigned* s = L.state + (size_t)lod * L.stride + v;
    if (*s == 0u) *s = kWanted;
}

// Copy one voxel's n triangles from the host bytes at src (any alignment: the
// objects follow a one-byte header) into the device records dst, 32 at a
// time.  For each 32: the 16-byte chunks that hold their 9 x 32 coordinate
// words and (further on, after all n triangles) their 2 x 32 bound words are
// loaded with every load in flight at once, land in shared memory as they
// are, and each lane then assembles its triangle's words with a funnel
// shift.  Every chunk read holds a byte of the voxel's block, so it lies on a
// page of the registered buffer.
__device__ void copy_voxel(uintptr_t src, uint32_t n, float4* __restrict__ dst, uint32_t* st) {
    const int lane = threadIdx.x & 31;
    uint32_t* sT = st;
    uint32_t* sH = st + kStageT;
    const unsigned sh = (unsigned)(src & 3) * 8;  // 36 and 8 keep the byte alignment
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t m = min(32u, n - c0);
        const uintptr_t pT = src + 36 * (uintptr_t)c0, pH = src + 36 * (uintptr_t)n + 8 * (uintptr_t)c0;
        const uintptr_t aT = pT & ~uintptr_t(15), aH = pH & ~uintptr_t(15);
        const uint32_t nT = (uint32_t)((((pT + 36 * (uintptr_t)m + 15) & ~uintptr_t(15)) - aT) >> 4);
        const uint32_t nH = (uint32_t)((((pH + 8 * (uintptr_t)m + 15) & ~uintptr_t(15)) - aH) >> 4);
        const uint4* QT = reinterpret_cast<const uint4*>(aT);
        const uint4* QH = reinterpret_cast<const uint4*>(aH);
        uint4 qT[3], qH;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t i = 32 * k + lane;
            qT[k] = i < nT ? QT[i] : make_uint4(0u, 0u, 0u, 0u);
        }
        qH = (uint32_t)lane < nH ? QH[lane] : make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();  // the previous round's lanes are done with the stage
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t i = 32 * k + lane;
            if (i < nT) reinterpret_cast<uint4*>(sT)[i] = qT[k];
        }
        if ((uint32_t)lane < nH) reinterpret_cast<uint4*>(sH)[lane] = qH;
        __syncwarp();
        if ((uint32_t)lane < m) {
            // word j of this triangle: bytes [pT - aT + 36 lane + 4 j, +4) of sT
            const uint32_t wT = (uint32_t)((pT - aT) >> 2) + 9 * lane;
            const uint32_t wH = (uint32_t)((pH - aH) >> 2) + 2 * lane;
            uint32_t f[9], h[2];
#pragma unroll
            for (int j = 0; j < 9; ++j) f[j] = sh ? __funnelshift_r(sT[wT + j], sT[wT + j + 1], sh) : sT[wT + j];
#pragma unroll
            for (int j = 0; j < 2; ++j) h[j] = sh ? __funnelshift_r(sH[wH + j], sH[wH + j + 1], sh) : sH[wH + j];
            float4* r = dst + 3 * (size_t)(c0 + lane);
            r[0] = make_float4(__uint_as_float(f[0]), __uint_as_float(f[1]), __uint_as_float(f[2]),
                               __uint_as_float(h[0]));
            r[1] = make_float4(__uint_as_float(f[3]), __uint_as_float(f[4]), __uint_as_float(f[5]),
                               __uint_as_float(h[1]));
            r[2] = make_float4(__uint_as_float(f[6]), __uint_as_float(f[7]), __uint_as_float(f[8]), 0.f);
        }
    }
}

// mark the voxels every item names at LOD index lod (one thread per item)
__global__ void k_mark_items(const RefineItem* __restrict__ items, const unsigned* n_dev, long n_host, int lod,
                             LazyTile A, LazyTile B) {
    const long n = n_dev ? (long)*n_dev : n_host;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const RefineItem it = items[i];
        if (A.on && it.a_cnt) mark(A, lod, last_le(A.vtri[lod], A.n_vox + 1, it.a_off));
        if (B.on && it.b_cnt) mark(B, lod, last_le(B.vtri[lod], B.n_vox + 1, it.b_off));
    }
}

// mark both voxels of every live voxel pair of an undecided object pair
__global__ void k_mark_pairs(const uint8_t* __restrict__ valive, const int* __restrict__ vpair,
                             const uint8_t* pstat, const int* __restrict__ vpa, const int* __restrict__ vpb,
                             int64_t V, int lod, LazyTile A, LazyTile B) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
        if (!valive[v] || pstat[vpair[v]] != 0) continue;
        if (A.on) mark(A, lod, vpa[v]);
        if (B.on) mark(B, lod, vpb[v]);
    }
}

// Fetch every voxel of tile A, then of tile B (skipped when it is A itself),
// whose state at LOD index lod is kWanted (ALL: also 0), and set it to 1.
// Lanes look at 32 voxels at a time and work out where the wanted ones sit
// in the host bytes; the warp then copies them one after the other.
template <bool ALL>
__global__ void __launch_bounds__(kFetchWarps * 32) k_fetch_marked(int lod, LazyTile A, LazyTile B) {
    __shared__ __align__(16) uint32_t stage[kFetchWarps][kStageWords];
    uint32_t* st = stage[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const long na = A.on ? A.n_vox : 0;
    const long nb = B.on && !(A.on && A.state == B.state) ? B.n_vox : 0;
    const long total = na + nb;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long bytes_a = 0, bytes_b = 0;
    for (long base = (((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < total; base += warps * 32) {
        const long g = base + lane;
        const bool in_a = g < na;
        const LazyTile& T = in_a ? A : B;
        const long v = in_a ? g : g - na;
        bool want = false;
        uint32_t off = 0, cnt = 0;
        uintptr_t src = 0;
        if (g < total) {
            unsigned* sp = T.state + (size_t)lod * T.stride + v;
            const unsigned sv = *sp;
            if (sv == kWanted || (ALL && sv == 0u)) {
                off = T.vtri[lod][v];
                cnt = T.vtri[lod][v + 1] - off;
                if (cnt) src = voxel_src(T, lod, v, off);
                want = true;
                *sp = 1u;  // read by later launches only
            }
        }
        unsigned m = __ballot_sync(0xffffffffu, want && cnt > 0);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const unsigned long long s64 = __shfl_sync(0xffffffffu, (unsigned long long)src, l);
            const uint32_t o = __shfl_sync(0xffffffffu, off, l), c = __shfl_sync(0xffffffffu, cnt, l);
            const bool ia = __shfl_sync(0xffffffffu, in_a ? 1 : 0, l) != 0;
            copy_voxel((uintptr_t)s64, c, (ia ? A : B).tri[lod] + 3 * (size_t)o, st);
            if (ia) bytes_a += 44ull * c;
            else bytes_b += 44ull * c;
        }
    }
    if (lane == 0) {
        if (bytes_a) atomicAdd(A.bytes, bytes_a);
        if (bytes_b) atomicAdd(B.bytes, bytes_b);
    }
}

int mark_grid(int64_t n, int num_sms) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms * 8));
}

cudaError_t launch_fetch_marked(int lod, const LazyTile& a, const LazyTile& b, int num_sms, cudaStream_t s,
                                bool all = false) {
    const long total = (a.on ? a.n_vox : 0) + (b.on ? b.n_vox : 0);
    if (total <= 0) return cudaSuccess;
    const long need = (total + 32 * kFetchWarps - 1) / (32 * kFetchWarps);
    const int blocks = (int)std::max(1L, std::min<long>(need, (long)num_sms * 8));
    if (all) k_fetch_marked<true><<<blocks, kFetchWarps * 32, 0, s>>>(lod, a, b);
    else k_fetch_marked<false><<<blocks, kFetchWarps * 32, 0, s>>>(lod, a, b);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_prefetch_pairs(const uint8_t* valive, const int* vpair, const uint8_t* pstat, const int* vpa,
                                  const int* vpb, int64_t V, int lod, const LazyTile& a, const LazyTile& b,
                                  int num_sms, cudaStream_t s) {
    if ((!a.on && !b.on) || V <= 0) return cudaSuccess;
    k_mark_pairs<<<mark_grid(V, num_sms), 256, 0, s>>>(valive, vpair, pstat, vpa, vpb, V, lod, a, b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_fetch_marked(lod, a, b, num_sms, s);
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
    const int blocks = n_dev ? num_sms * 8 : mark_grid(n_host, num_sms);
    k_mark_items<<<blocks, 256, 0, s>>>(items, n_dev, n_host, lod, a, b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_fetch_marked(lod, a, b, num_sms, s);
}

cudaError_t launch_fetch_all(const LazyTile& t, int num_sms, cudaStream_t s) {
    if (!t.on || t.n_vox == 0) return cudaSuccess;
    for (int l = 0; l < kNumLods; ++l) {
        const cudaError_t e = launch_fetch_marked(l, t, LazyTile{}, num_sms, s, true);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace tdp
