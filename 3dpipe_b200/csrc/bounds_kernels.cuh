// bounds_kernels.cuh -- launchers of bounds_kernels.cu used by host code.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace tdp {
// (proxy, hausdorff) of n triangle records -> out[2i], out[2i+1]
cudaError_t launch_gather_bounds(const float4* tri, size_t n, float* out, cudaStream_t s);
}  // namespace tdp
