// exact_kernels.cuh -- FP64 LOD-100 distances of the reported object pairs.
#pragma once
#include <cuda_runtime.h>

#include "ctx.cuh"
#include "fetch_kernels.cuh"
#include "join_kernels.cuh"
#include "storage/dev_tile.h"

namespace tdp {

struct ExactInfo {
    long items = 0;      // LOD-100 voxel pairs refined in FP32 (box gap within the pair's upper bound)
    long f64_items = 0;  // of those, evaluated in FP64 (FP32 minimum within the error band of the best)
    int launches = 0;
    double max_rel_err32 = 0;  // max |FP32 object minimum - FP64 distance| / max(distance, 1)
    double phase_ms[4] = {0, 0, 0, 0};  // upper bounds, candidates, FP32 pass, FP64 pass (device time)
    unsigned long long full_evals = 0;  // triangle pairs the FP32 pass evaluated fully
    long dropped_items = 0;  // FP32 pass items dropped by the refine's item-level test
    long below_items = 0;    // FP32 pass items with a triangle pair below their preset
};

// For every object pair with pstat == kReported: the exact minimum triangle
// distance at LOD 100, in double, written to pexact[p] (other pairs, and a
// reported pair without any LOD-100 triangles: values >= 1e300).
// pmx_valid: the pairs' upper bounds pmx bound the LOD-100 distance (true at
// Hausdorff level 2; levels 0 and 1 widen by nothing or by proxy-Hausdorff).
// lz1 / lz2: the tiles' fetch views (attached tiles fetch the LOD-100 voxels
// that the stage refines; resident tiles: raw == nullptr).
int exact_distances(tdp_ctx* ctx, const JoinDev& d, const tdp_tile* t1, const tdp_tile* t2, bool pmx_valid,
                    double* pexact, ExactInfo& info, const LazyTile& lz1, const LazyTile& lz2);

}  // namespace tdp
