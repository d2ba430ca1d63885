// attach_kernels.cu -- the metadata pass of tdp_tile_attach on the GPU.
//
// An attached tile stays in page-locked host memory; the device needs its
// metadata: per voxel the box and core (3 float4) and the triangle count at
// every LOD (as prefix arrays), per object the Hausdorff values, voxel range,
// box and transform (the reference's RAW reader, HiMesh_Wrapper(char*, id, RAW),
// src/spatial/himesh_wrapper.cpp:48-83, reads the same fields).  After the
// host's walk over the size fields (walk_raw_dt) has found every object's
// record, one warp per object reads that object's metadata block -- about 1.5
// KB for a nucleus, every 170 KB of the file -- straight from the mapped host
// bytes, instead of a host pass over them followed by copies of its results.
// The blocks follow a one-byte header, so they are read as the 16-byte
// aligned chunks that hold them, all of a window's loads in flight at once,
// and realigned with a funnel shift in shared memory; every chunk read holds
// bytes of the record, which the walk checked lies inside the buffer.
//
// Validation: every check the host parser makes on these fields (voxel boxes
// not inverted, each LOD range inside the object's data block, 4-byte
// aligned, at most 2^24 triangles) plus the writer's layout that attach
// requires (each voxel's triangles, LOD by LOD and voxel by voxel, with nothing
// in between) is made on the device; a failure only flags the lowest failing
// object, and the caller then parses the tile on the host, which reports the
// first error in file order with its usual message.
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "attach_kernels.cuh"
#include "common.cuh"

namespace tdp {
namespace {

constexpr int kWarps = 8;
constexpr int kVoxWords = 29;  // 9 floats + 5 x (offset, count) as u64
constexpr int kChunkVox = 32;  // voxels per warp and round (one per lane)
constexpr int kHdWords = 2 * kNumLods;
// words staged per window: 2 lead words (the voxel count before the
// Hausdorff values, first window), the tables, the transform and 2 tail
// words (the next object's data size, last window)
constexpr int kStage = 2 + kHdWords + kChunkVox * kVoxWords + 3 + 2;

constexpr int kChunks = (4 * kStage + 30) / 16 + 1;  // 16-byte chunks a window spans, at most
constexpr int kChunkLoads = (kChunks + 31) / 32;      // per lane
constexpr int kWordLoads = (kStage + 31) / 32;        // per lane
constexpr int kStageAlloc = 4 * kChunks + 8;          // words of a warp's stage (16-byte rows)

// st[i] = the 32-bit value at byte address p + 4 i, for i < cnt (p of any
// alignment).  The bytes are read as the 16-byte aligned chunks that hold
// them -- every chunk holds a byte of the values, so it lies on a page they
// occupy -- with every load of the window issued before any is used (a
// zero-copy read of host memory takes microseconds, and more loads in flight
// per warp lift the rate from ~33 to ~49 GB/s); the chunks land in the stage
// as they are and are realigned in place through registers.
__device__ __forceinline__ void stage_chunks(uintptr_t p, uint32_t cnt, int lane, uint32_t* st) {
    const uintptr_t a0 = p & ~uintptr_t(15);
    const uint32_t nq = (uint32_t)((((p + 4 * (uintptr_t)cnt + 15) & ~uintptr_t(15)) - a0) >> 4);
    const uint4* Q = reinterpret_cast<const uint4*>(a0);
    uint4 q[kChunkLoads];
#pragma unroll
    for (int k = 0; k < kChunkLoads; ++k) {
        const uint32_t i = 32 * k + lane;
        q[k] = i < nq ? Q[i] : make_uint4(0u, 0u, 0u, 0u);
    }
    uint4* S4 = reinterpret_cast<uint4*>(st);
#pragma unroll
    for (int k = 0; k < kChunkLoads; ++k) {
        const uint32_t i = 32 * k + lane;
        if (i < nq) S4[i] = q[k];
    }
    __syncwarp();
    const uint32_t off = (uint32_t)(p - a0), w0 = off >> 2;
    const unsigned sh = (off & 3) * 8;
    uint32_t v[kWordLoads];
#pragma unroll
    for (int k = 0; k < kWordLoads; ++k) {
        const uint32_t i = 32 * k + lane;  // w0 + i + 1 <= 4 kChunks + 3 < kStageAlloc
        v[k] = i < cnt ? (sh ? __funnelshift_r(st[w0 + i], st[w0 + i + 1], sh) : st[w0 + i]) : 0u;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kWordLoads; ++k) {
        const uint32_t i = 32 * k + lane;
        if (i < cnt) st[i] = v[k];
    }
}

// sr.on: the records are placed at the first record's stride instead of
// walked, so every object's voxel count (the 8 bytes before its Hausdorff
// values) and the next object's data size (the 8 bytes after its transform)
// are checked against the first object's, read with the windows they border
__global__ void __launch_bounds__(kWarps * 32) k_parse_tables(const uint8_t* __restrict__ raw,
                                                              const AttachRec* __restrict__ recs, long n_obj,
                                                              AttachOut o, AttachStride sr) {
    const bool strided = sr.on != 0;
    const uint64_t data_size0 = sr.first.data_size;
    __shared__ __align__(16) uint32_t stage[kWarps][kStageAlloc];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t* st = stage[w];
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long ob = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; ob < n_obj; ob += nw) {
        const AttachRec r = strided ? AttachRec{sr.first.data_off + (uint64_t)ob * sr.stride, sr.first.data_size,
                                                sr.first.meta + (uint64_t)ob * sr.stride, sr.first.vnum,
                                                (uint32_t)ob * sr.first.vnum}
                                    : recs[ob];
        const uintptr_t base = reinterpret_cast<uintptr_t>(raw) + r.meta;
        const uint64_t xw = kHdWords + (uint64_t)r.vnum * kVoxWords;  // first transform word
        bool bad = false;
        float lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY, hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
        unsigned long long tris[kNumLods] = {0, 0, 0, 0, 0};
        float xf = 0.f;
        // windows of the metadata block: [Hausdorff values] 32 voxels [transform]
        for (uint32_t c0 = 0; c0 < r.vnum; c0 += kChunkVox) {
            const uint32_t m = min((uint32_t)kChunkVox, r.vnum - c0);
            const bool last = c0 + m == r.vnum;
            const uint64_t ws = c0 == 0 ? 0 : kHdWords + (uint64_t)c0 * kVoxWords;
            const uint64_t we = kHdWords + (uint64_t)(c0 + m) * kVoxWords + (last ? 3 : 0);
            const uint32_t lead = strided && c0 == 0 ? 2u : 0u;
            const uint32_t tail = strided && last && ob + 1 < n_obj ? 2u : 0u;
            __syncwarp();
            stage_chunks(base + 4 * ws - 4 * lead, (uint32_t)(we - ws) + lead + tail, lane, st);
            __syncwarp();
            const uint32_t* S = st + lead;  // S[i]: word ws + i of the block
            if (lead && ((uint64_t)st[0] | ((uint64_t)st[1] << 32)) != r.vnum) bad = true;
            if (tail && ((uint64_t)S[we - ws] | ((uint64_t)S[we - ws + 1] << 32)) != data_size0) bad = true;
            if (c0 == 0 && lane < kHdWords) {  // object Hausdorff values: 5 x (hausdorff, proxy)
                const float v = __uint_as_float(S[lane]);
                if (lane & 1) o.obj_phd[ob * kNumLods + (lane >> 1)] = v;
                else o.obj_hd[ob * kNumLods + (lane >> 1)] = v;
            }
            if (last && lane < 3) xf = __uint_as_float(S[xw - ws + lane]);
            if (lane < m) {
                const uint32_t* q = S + (kHdWords + (uint64_t)(c0 + lane) * kVoxWords - ws);
                const uint32_t v = r.vox0 + c0 + lane;
                float b[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) b[k] = __uint_as_float(q[k]);
                if (!(b[0] <= b[3]) || !(b[1] <= b[4]) || !(b[2] <= b[5])) bad = true;
                o.vox[3 * (size_t)v + 0] = make_float4(b[0], b[1], b[2], 0.f);
                o.vox[3 * (size_t)v + 1] = make_float4(b[3], b[4], b[5], 0.f);
                o.vox[3 * (size_t)v + 2] = make_float4(b[6], b[7], b[8], 0.f);
                lo0 = fminf(lo0, b[0]); lo1 = fminf(lo1, b[1]); lo2 = fminf(lo2, b[2]);
                hi0 = fmaxf(hi0, b[3]); hi1 = fmaxf(hi1, b[4]); hi2 = fmaxf(hi2, b[5]);
#pragma unroll
                for (int l = 0; l < kNumLods; ++l) {
                    const uint64_t off = (uint64_t)q[9 + 4 * l] | ((uint64_t)q[10 + 4 * l] << 32);
                    const uint64_t cnt = (uint64_t)q[11 + 4 * l] | ((uint64_t)q[12 + 4 * l] << 32);
                    if (cnt > (1u << 24) || (off & 3) || off > r.data_size || cnt * 44 > r.data_size - off) {
                        bad = true;
                        o.vtri[l][v + 1] = 0;
                        o.off4[l][v] = 0;
                    } else {
                        o.vtri[l][v + 1] = (uint32_t)cnt;  // the inclusive scan turns counts into the prefix
                        o.off4[l][v] = (uint32_t)(off >> 2);
                        tris[l] += cnt;
                    }
                }
                o.vobj[v] = (uint32_t)ob;
            }
        }
        // object box (the union of the voxel boxes, as the reference reader
        // forms it), transform, voxel range, data block offset
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            lo0 = fminf(lo0, __shfl_xor_sync(0xffffffffu, lo0, s));
            lo1 = fminf(lo1, __shfl_xor_sync(0xffffffffu, lo1, s));
            lo2 = fminf(lo2, __shfl_xor_sync(0xffffffffu, lo2, s));
            hi0 = fmaxf(hi0, __shfl_xor_sync(0xffffffffu, hi0, s));
            hi1 = fmaxf(hi1, __shfl_xor_sync(0xffffffffu, hi1, s));
            hi2 = fmaxf(hi2, __shfl_xor_sync(0xffffffffu, hi2, s));
#pragma unroll
            for (int l = 0; l < kNumLods; ++l) tris[l] += __shfl_xor_sync(0xffffffffu, tris[l], s);
        }
        if (lane < 3) o.boxes[6 * n_obj + 3 * ob + lane] = xf;
        if (lane == 0) {
            float* bx = o.boxes + 6 * ob;
            bx[0] = lo0; bx[1] = lo1; bx[2] = lo2; bx[3] = hi0; bx[4] = hi1; bx[5] = hi2;
            o.obj_vox[ob] = r.vox0;
            o.data_off[ob] = r.data_off;
#pragma unroll
            for (int l = 0; l < kNumLods; ++l)
                if (tris[l]) atomicAdd(o.n_tris + l, tris[l]);
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicMin(o.first_bad, (unsigned long long)ob);
    }
}

// The writer's layout: the (LOD l, voxel v) block of object o starts 44 bytes
// times the object's triangles before it in LOD-then-voxel order into the data
// block (what the fetch kernels compute from the prefix arrays).
__global__ void k_check_layout(AttachOut o, long n_vox) {
    const long total = (long)kNumLods * n_vox;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int l = (int)(i / n_vox);
        const long v = i - (long)l * n_vox;
        const uint32_t ob = o.vobj[v];
        const uint32_t vb = o.obj_vox[ob], ve = o.obj_vox[ob + 1];
        uint64_t before = o.vtri[l][v] - o.vtri[l][vb];
        for (int k = 0; k < l; ++k) before += o.vtri[k][ve] - o.vtri[k][vb];
        if ((uint64_t)o.off4[l][v] != 11 * before) atomicMin(o.first_bad, (unsigned long long)ob);
    }
}

}  // namespace

cudaError_t launch_attach_tables(const uint8_t* raw_dev, const AttachRec* recs, long n_obj, long n_vox,
                                 const AttachOut& out, void* scan_tmp, size_t& scan_bytes, int num_sms,
                                 cudaStream_t s, const AttachStride& st) {
    if (!scan_tmp) {  // size query for the scans
        size_t b = 0;
        const cudaError_t e =
            cub::DeviceScan::InclusiveSum(nullptr, b, out.vtri[0] + 1, out.vtri[0] + 1, (int)n_vox, s);
        scan_bytes = b;
        return e;
    }
    if (n_obj <= 0) return cudaSuccess;
    for (int l = 0; l < kNumLods; ++l) {
        const cudaError_t e = cudaMemsetAsync(out.vtri[l], 0, sizeof(uint32_t), s);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (int)std::max<long>(1, std::min<long>((n_obj + kWarps - 1) / kWarps, (long)num_sms * 16));
    k_parse_tables<<<blocks, kWarps * 32, 0, s>>>(raw_dev, recs, n_obj, out, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    for (int l = 0; l < kNumLods; ++l) {  // in place: counts at [1, n_vox] become the prefix
        size_t b = scan_bytes;
        e = cub::DeviceScan::InclusiveSum(scan_tmp, b, out.vtri[l] + 1, out.vtri[l] + 1, (int)n_vox, s);
        if (e != cudaSuccess) return e;
    }
    const long total = (long)kNumLods * n_vox;
    const int cb = (int)std::max<long>(1, std::min<long>((total + 255) / 256, (long)num_sms * 16));
    k_check_layout<<<cb, 256, 0, s>>>(out, n_vox);
    return cudaGetLastError();
}

}  // namespace tdp
