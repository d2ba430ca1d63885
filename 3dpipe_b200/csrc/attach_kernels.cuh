// attach_kernels.cuh -- the metadata pass of tdp_tile_attach on the GPU (see
// attach_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "storage/dt_format.h"

namespace tdp {

// One object as the host walk found it (walk_raw_dt), plus its first voxel.
struct AttachRec {
    uint64_t data_off;   // byte offset of the data block in the tile buffer
    uint64_t data_size;  // bytes of the data block
    uint64_t meta;       // byte offset of the object Hausdorff values (after vnum)
    uint32_t vnum;       // voxels
    uint32_t vox0;       // first voxel of the object in the tile
};

// Records placed at a fixed stride instead of walked (a tile of equal-size
// records): object o is `first` moved o * stride bytes on, its first voxel
// o * first.vnum.  on == 0: the records come from the uploaded array.
struct AttachStride {
    int on;
    uint64_t stride;
    AttachRec first;
};

// Where the pass writes (all device memory).
struct AttachOut {
    float4* vox;                      // [3 n_vox] (low, 0) (high, 0) (core, 0)
    uint32_t* obj_vox;                // [n_obj + 1] (entry n_obj set by the caller)
    float* obj_hd;                    // [5 n_obj]
    float* obj_phd;                   // [5 n_obj]
    float* boxes;                     // [9 n_obj]: 6 n_obj box floats, then 3 n_obj transform floats
    uint64_t* data_off;               // [n_obj]
    uint32_t* vtri[kNumLods];         // [n_vox + 1] each: counts, then their prefix
    uint32_t* off4[kNumLods];         // [n_vox] each: declared data-block offset / 4 (layout check)
    uint32_t* vobj;                   // [n_vox] object of each voxel
    unsigned long long* n_tris;       // [5] triangles per LOD (zeroed by the caller)
    unsigned long long* first_bad;    // lowest failing object (~0 when none; set by the caller)
};

// Parse the voxel tables of n_obj objects from raw_dev (the device view of the
// page-locked tile bytes), scan the counts into vtri, check the layout.  Call
// first with scan_tmp == nullptr to learn scan_bytes.
// st.on: the records are placed at the first record's stride (no walk, recs
// unused); each object's voxel count and the next object's data size are
// then checked against the first object's, and a difference flags the
// object in first_bad (the caller walks the tile on the host).
cudaError_t launch_attach_tables(const uint8_t* raw_dev, const AttachRec* recs, long n_obj, long n_vox,
                                 const AttachOut& out, void* scan_tmp, size_t& scan_bytes, int num_sms,
                                 cudaStream_t s, const AttachStride& st = AttachStride{});

}  // namespace tdp
