// tile_kernels.cuh -- the RAW triangle unpack kernel, shared by tile upload
// (csrc/tile.cu) and the serving arenas (src/serve/server.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tdp {

struct UnpackSeg {
    uint64_t src;      // byte offset of the segment's triangles in the staging buffer
    uint32_t dst;      // first destination triangle in tri[lod]
    uint32_t cnt_lod;  // count (low 24 bits) | lod << 24
};

// One warp per segment: the segment's RAW triangles (9 floats each, then 2
// Hausdorff floats each) become 48-byte records at tri[lod][dst...].  Every
// segment's src must be 4-byte aligned in `raw` (checked by the callers).
cudaError_t launch_unpack(const uint8_t* raw, const UnpackSeg* segs, int nseg, float4* const* tri, int num_sms,
                          cudaStream_t s);

}  // namespace tdp
