// noalloc.cu -- tdp_refine_batch_noalloc: the batched refine for callers that
// cannot allocate device memory.
//
// Who needs it: code that owns no device allocator of its own, for example a
// plugin running inside a host application that has already claimed all of the
// GPU's memory through its own pool, a process held to a fixed device-memory
// budget, or a latency-critical loop that must not call cudaMalloc (which can
// block until the whole device is idle).  tdp_refine_batch cannot serve them:
// it keeps its buffers in a context it allocates.  This entry point takes
// device pointers for every input and output and keeps its own working memory
// (packed triangles, work items, per-pair results, counters) in one
// file-scope __device__ array of fixed size, so it never calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// Limits: at most kNoAllocMaxTris triangles and kNoAllocMaxPairs voxel pairs
// per call (the array holds kScratchBytes = 14,680,320 bytes, 14.0 MiB; every
// GPU that loads this library keeps it until the process exits).  Larger
// batches are rejected with an error.
//
// Kernel: the tuned refine in its configuration 0 (eager staging, A chunk of
// 64 triangles, 3 CTAs per SM) -- a call has no context, so no autotuner pick
// applies.  Its minima equal those of every other tuned configuration.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress while that device is current, and caches it; the
// first launch of the tuned kernel in a process also raises its dynamic
// shared-memory limit (cudaFuncSetAttribute).  Make that first call before any
// stream capture begins.  All calls on a device share the one array and each
// call overwrites it, so calls whose work can overlap on the GPU (other
// streams, other host threads) race: serialise them.
#include <float.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "refine.cuh"
#include "tdp.h"

namespace tdp {
namespace {

constexpr uint32_t kNoAllocMaxTris = 1u << 18;   // 262,144 triangles
constexpr uint32_t kNoAllocMaxPairs = 1u << 16;  // 65,536 voxel pairs
constexpr size_t kOffCounters = 0;               // work counter, full-evaluation counter
constexpr size_t kOffItems = 256;
constexpr size_t kOffRes = kOffItems + (size_t)kNoAllocMaxPairs * sizeof(RefineItem);
constexpr size_t kOffTris = kOffRes + (size_t)kNoAllocMaxPairs * sizeof(float4);
constexpr size_t kScratchBytes = kOffTris + (size_t)kNoAllocMaxTris * kTriF4 * sizeof(float4);

static __device__ __align__(256) unsigned char g_refine_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

int report(char* err, size_t cap, int code, const std::string& msg) {
    if (err && cap) {
        std::strncpy(err, msg.c_str(), cap - 1);
        err[cap - 1] = 0;
    }
    return code;
}

__device__ __forceinline__ bool item_ok(const size_t* os, uint32_t i, size_t n_tris) {
    const size_t o1 = os[4 * i], n1 = os[4 * i + 1], o2 = os[4 * i + 2], n2 = os[4 * i + 3];
    return o1 <= n_tris && n1 <= n_tris - o1 && o2 <= n_tris && n2 <= n_tris - o2;
}

// Zero the counters, pack the triangles into 48-byte records and convert the
// (off1, n1, off2, n2) rows into work items; a row that points outside the
// batch becomes an empty item (no read past the inputs) and gets NaN results.
__global__ void noalloc_prepare_kernel(const float* __restrict__ data, const float* __restrict__ hd, uint32_t n_tris,
                                       const size_t* __restrict__ os, uint32_t n_pairs, unsigned char* scratch) {
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(scratch + kOffCounters);
    RefineItem* items = reinterpret_cast<RefineItem*>(scratch + kOffItems);
    float4* tri = reinterpret_cast<float4*>(scratch + kOffTris);
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
    if (tid < 32) counters[tid] = 0ull;
    for (size_t i = tid; i < n_tris; i += stride) {
        const float* d = data + 9 * i;
        const float ph = hd ? hd[2 * i] : 0.f, h = hd ? hd[2 * i + 1] : 0.f;
        tri[3 * i + 0] = make_float4(d[0], d[1], d[2], ph);
        tri[3 * i + 1] = make_float4(d[3], d[4], d[5], h);
        tri[3 * i + 2] = make_float4(d[6], d[7], d[8], 0.f);
    }
    for (size_t i = tid; i < n_pairs; i += stride)
        items[i] = item_ok(os, (uint32_t)i, n_tris)
                       ? RefineItem{(uint32_t)os[4 * i], (uint32_t)os[4 * i + 1], (uint32_t)os[4 * i + 2],
                                    (uint32_t)os[4 * i + 3]}
                       : RefineItem{0, 0, 0, 0};
}

__global__ void noalloc_finish_kernel(const float4* __restrict__ res, const size_t* __restrict__ os, uint32_t n_tris,
                                      uint32_t n_pairs, int with_hd, float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_pairs; i += (size_t)gridDim.x * blockDim.x) {
        if (!item_ok(os, (uint32_t)i, n_tris)) {
            out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = __int_as_float(0x7fc00000);
            continue;
        }
        const float4 r = res[i];
        out[3 * i] = r.x;
        out[3 * i + 1] = with_hd ? r.y : FLT_MAX;
        out[3 * i + 2] = with_hd ? r.z : FLT_MAX;
    }
}

}  // namespace
}  // namespace tdp

using namespace tdp;

extern "C" int tdp_refine_batch_noalloc(const float* data, const float* hausdorff, size_t element_num,
                                        const size_t* offset_size, uint32_t pair_num, float* out, void* stream,
                                        char* err, size_t err_cap) {
    if (pair_num == 0) return TDP_OK;
    if (!data || !offset_size || !out) return report(err, err_cap, TDP_ERR_ARG, "null device pointer");
    if (element_num == 0 || element_num > kNoAllocMaxTris)
        return report(err, err_cap, TDP_ERR_ARG,
                      "element_num " + std::to_string(element_num) + " outside 1.." + std::to_string(kNoAllocMaxTris) +
                          ": the allocation-free refine holds at most that many triangles per call");
    if (pair_num > kNoAllocMaxPairs)
        return report(err, err_cap, TDP_ERR_ARG,
                      "pair_num " + std::to_string(pair_num) + " exceeds " + std::to_string(kNoAllocMaxPairs) +
                          ", the most voxel pairs the allocation-free refine holds per call");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return report(err, err_cap, TDP_ERR_NODEV, "no current CUDA device");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_addr[dev]) {
            cudaError_t e = cudaGetSymbolAddress(&g_addr[dev], g_refine_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                return report(err, err_cap, TDP_ERR_CUDA,
                              std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            }
        }
        base = g_addr[dev];
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* scratch = (unsigned char*)base;
    const uint32_t n_tris = (uint32_t)element_num;
    int blocks = (int)std::min<size_t>(((size_t)std::max(n_tris, pair_num) + 255) / 256, (size_t)sms * 8);
    noalloc_prepare_kernel<<<blocks, 256, 0, s>>>(data, hausdorff, n_tris, offset_size, pair_num, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report(err, err_cap, TDP_ERR_CUDA, cudaGetErrorString(e));
    const float4* tri = reinterpret_cast<const float4*>(scratch + kOffTris);
    e = launch_refine_tuned(tri, tri, reinterpret_cast<const RefineItem*>(scratch + kOffItems), (int)pair_num,
                            reinterpret_cast<float4*>(scratch + kOffRes),
                            reinterpret_cast<unsigned*>(scratch + kOffCounters),
                            reinterpret_cast<unsigned long long*>(scratch + kOffCounters + 8), sms, 0, s);
    if (e != cudaSuccess) return report(err, err_cap, TDP_ERR_CUDA, cudaGetErrorString(e));
    blocks = (int)std::min<size_t>(((size_t)pair_num + 255) / 256, (size_t)sms * 8);
    noalloc_finish_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(scratch + kOffRes), offset_size,
                                                  n_tris, pair_num, hausdorff != nullptr, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return report(err, err_cap, TDP_ERR_CUDA, cudaGetErrorString(e));
    return TDP_OK;
}
