// dev_tile.h -- a tile resident in HBM (behind the opaque tdp_tile of the C ABI).
//
// Layout in device memory:
//   vox       3 float4 per voxel: (low xyz, 0) (high xyz, 0) (core xyz, 0)
//   obj_vox   [n_obj+1] first voxel of each object
//   obj_hd    [n_obj*5] object-level hausdorff per LOD, obj_phd proxy
//   tri[l]    3 float4 per triangle of LOD l (see csrc/common.cuh RefineItem),
//             grouped by voxel in voxel order
//   vtri[l]   [n_vox+1] first triangle of each voxel at LOD l
// The host keeps the parsed metadata (boxes, transforms, counts) for candidate
// generation and for the join driver.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "storage/dt_format.h"

namespace tdp {
// A uniform grid over a tile's object boxes or transform points, resident on
// the device (built once per tile, on first use by a join).
struct DevGrid {
    float lo[3] = {0, 0, 0};
    float cell = 1.f, slack = 0.f;
    int n[3] = {1, 1, 1};
    int64_t* start = nullptr;  // [cells + 1]
    int32_t* items = nullptr;
    bool ready = false;
};
}  // namespace tdp

struct tdp_tile {
    tdp::TileHost host;
    mutable tdp::DevGrid box_grid, point_grid;  // object candidate grids (lazily built)
    // device copy of the objects' boxes (6 floats each) then transforms (3
    // each), made on first use by candidate generation; boxes_n != n_obj
    // (or 0 after a serving-arena append) means stale
    mutable float* d_boxes = nullptr;
    mutable long boxes_n = 0;
    long n_obj = 0, n_vox = 0;
    float4* vox = nullptr;
    uint32_t* obj_vox = nullptr;
    float* obj_hd = nullptr;
    float* obj_phd = nullptr;
    float4* tri[tdp::kNumLods] = {};
    uint32_t* vtri[tdp::kNumLods] = {};
    tdp::HostVec<uint32_t> h_vtri[tdp::kNumLods];  // host copy of vtri
    size_t device_bytes = 0;
    size_t h2d_bytes = 0;  // bytes copied host -> device by the upload or attach itself
    double parse_ms = 0, alloc_ms = 0, meta_ms = 0, load_ms = 0;  // host time of the upload or attach
    int device = 0;
    // attached tiles (tdp_tile_attach): the triangles stay in page-locked host
    // memory and joins fetch the voxels they refine (csrc/fetch_kernels.cu)
    bool lazy_on = false;                       // joins fetch triangles (attached tiles, serving arenas)
    const uint8_t* lazy_raw = nullptr;          // device view of the host bytes (attached tiles; an arena's
                                                // lazy_data_off holds absolute device-view addresses)
    uint64_t* lazy_data_off = nullptr;          // [n_obj] byte offset of each object's data block
    unsigned* lazy_state = nullptr;             // [kNumLods * lazy_stride] 1 once the voxel's LOD is on the device
    long lazy_stride = 0;
    unsigned long long* lazy_bytes = nullptr;   // RAW bytes fetched so far
};
