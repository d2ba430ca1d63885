// fetch_kernels.cuh -- on-demand triangle fetch for attached tiles
// (tdp_tile_attach): the triangles stay in page-locked host memory and a join
// copies only the voxels its refine items touch, one LOD at a time.
//
// This is the reference's per-LOD staging of the voxels involved in a chunk
// (build_chunks_by_pair / packing_data_stream, src/join/KNNJoin.cpp:1473-1521,
// src/join/SpatialJoin.cpp:169-248) done by the GPU itself: each refine item
// names a whole voxel of each tile, a warp claims the voxel (a state word per
// voxel and LOD), reads its RAW bytes straight from the mapped host buffer and
// unpacks them into the tile's device records.  A voxel is fetched at most once
// per tile and LOD; the refine that follows reads device memory only.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "storage/dt_format.h"

struct tdp_tile;

namespace tdp {

struct LazyTile {
    bool on = false;                        // false: a resident tile, nothing to fetch
    const uint8_t* raw = nullptr;           // device view of the page-locked RAW bytes (or nullptr
                                            // when data_off holds absolute device-view addresses)
    const uint64_t* data_off = nullptr;     // [n_obj] where each object's data block starts
    const uint32_t* obj_vox = nullptr;      // [n_obj + 1]
    const uint32_t* vtri[kNumLods] = {};    // [n_vox + 1] first triangle of each voxel
    float4* tri[kNumLods] = {};             // device records
    unsigned* state = nullptr;              // [kNumLods * stride] 0 = not fetched, 1 = fetched (or resident)
    long stride = 0;                        // state entries per LOD (>= n_vox)
    unsigned long long* bytes = nullptr;    // RAW bytes fetched (counter)
    long n_vox = 0, n_obj = 0;
};

// the device view of a tile (on == false for a resident tile)
LazyTile lazy_view(const tdp_tile* t);

// fetch, for every item of `items` (n_dev: count in device memory, else
// n_host), the voxels it names at LOD index lod, for each attached side
cudaError_t launch_fetch_items(const RefineItem* items, const unsigned* n_dev, long n_host, int lod,
                               const LazyTile& a, const LazyTile& b, int num_sms, cudaStream_t s);
// fetch every voxel of every LOD of an attached tile
cudaError_t launch_fetch_all(const LazyTile& t, int num_sms, cudaStream_t s);
// prefetch, at LOD index lod, both voxels of every voxel pair v < V that is
// alive and whose object pair is undecided (valive[v], pstat[vpair[v]] == 0):
// a superset of the next LOD's refine items, run on a second stream beside
// the current LOD's refine.  The flags may change meanwhile; a voxel that is
// missed here is fetched by that LOD's own launch_fetch_items.
cudaError_t launch_prefetch_pairs(const uint8_t* valive, const int* vpair, const uint8_t* pstat, const int* vpa,
                                  const int* vpb, int64_t V, int lod, const LazyTile& a, const LazyTile& b,
                                  int num_sms, cudaStream_t s);

}  // namespace tdp
