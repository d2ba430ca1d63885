// serve_kernels.cu -- the serving arenas' commit kernel (see serve_kernels.cuh).
#include <algorithm>

#include "serve_kernels.cuh"

namespace tdp {
namespace {

struct Off {
    uint32_t t0[kNumLods];
};

__global__ void k_arena_commit(ArenaMeta m, ArenaDst d, long n, long nv, long o0, long v0, Off t) {
    const long stride = (long)gridDim.x * blockDim.x;
    const long nvox = 3 * nv, nobj = n, nhd = n * kNumLods;
    const long total = nvox + nobj + 2 * nhd + 2 * (long)kNumLods * nv + n;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        long k = i;
        if (k < nvox) { d.vox[3 * v0 + k] = m.vox[k]; continue; }
        k -= nvox;
        if (k < nobj) { d.obj_vox[o0 + 1 + k] = (uint32_t)v0 + m.obj_vox[k + 1]; continue; }
        k -= nobj;
        if (k < nhd) { d.obj_hd[o0 * kNumLods + k] = m.obj_hd[k]; continue; }
        k -= nhd;
        if (k < nhd) { d.obj_phd[o0 * kNumLods + k] = m.obj_phd[k]; continue; }
        k -= nhd;
        if (k < (long)kNumLods * nv) {
            const int l = (int)(k / nv);
            const long v = k - (long)l * nv;
            d.vtri[l][v0 + 1 + v] = t.t0[l] + m.vtri[l][v + 1];
            continue;
        }
        k -= (long)kNumLods * nv;
        if (k < (long)kNumLods * nv) {  // fetch state: 0 = to fetch, 1 = unpacked from staging
            const int l = (int)(k / nv);
            const long v = k - (long)l * nv;
            d.state[(size_t)l * d.stride + v0 + v] = m.fetched ? 0u : 1u;
            continue;
        }
        k -= (long)kNumLods * nv;
        d.data_off[o0 + k] = m.data_abs[k];
    }
}

}  // namespace

cudaError_t launch_arena_commit(const ArenaMeta& m, const ArenaDst& d, long n, long nv, long o0, long v0,
                                const uint32_t* t0, int num_sms, cudaStream_t s) {
    const long total = 3 * nv + n + 2 * n * kNumLods + 2 * (long)kNumLods * nv + n;
    if (total <= 0) return cudaSuccess;
    Off t;
    for (int l = 0; l < kNumLods; ++l) t.t0[l] = t0[l];
    const int blocks = (int)std::min<long>((total + 255) / 256, (long)num_sms * 8);
    k_arena_commit<<<blocks, 256, 0, s>>>(m, d, n, nv, o0, v0, t);
    return cudaGetLastError();
}

}  // namespace tdp
