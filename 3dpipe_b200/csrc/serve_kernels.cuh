// serve_kernels.cuh -- device side of the serving arenas (src/serve/server.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "storage/dt_format.h"

namespace tdp {

// A request's metadata in request-local offsets, staged next to its RAW
// bytes; the commit kernel adds the arena's offsets while writing it into the
// arena (so appending needs no host-to-device copy of its own).
struct ArenaMeta {
    const float4* vox;          // [3 nv] voxel records
    const uint32_t* obj_vox;    // [n + 1] local first voxel of each object
    const float* obj_hd;        // [n * kNumLods]
    const float* obj_phd;       // [n * kNumLods]
    const uint32_t* vtri[kNumLods];  // [nv + 1] local first triangle of each voxel
    const uint64_t* data_abs;   // [n] device-view address of each object's data block (fetched requests)
    unsigned fetched;           // 1: the join fetches the request's triangles from its own buffer
};

struct ArenaDst {
    float4* vox;
    uint32_t* obj_vox;
    float* obj_hd;
    float* obj_phd;
    uint32_t* vtri[kNumLods];
    uint64_t* data_off;  // the arena's per-object data-block addresses
    unsigned* state;     // the arena's fetch state, kNumLods planes of `stride` voxels
    long stride;
};

// Write n objects / nv voxels of `m` at object o0, voxel v0, triangle t0[l].
cudaError_t launch_arena_commit(const ArenaMeta& m, const ArenaDst& d, long n, long nv, long o0, long v0,
                                const uint32_t* t0, int num_sms, cudaStream_t s);

}  // namespace tdp
