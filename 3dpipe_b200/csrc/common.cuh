// common.cuh -- shared device-side definitions for the tdp library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

namespace tdp {

// One refine work item: a voxel pair at one LOD.  Offsets index triangles
// (3 float4 records each) in the A-side and B-side triangle arrays.
struct RefineItem {
    uint32_t a_off, a_cnt, b_off, b_cnt;
};

// Triangle record in HBM: 48 bytes, 16-byte aligned, loadable as 3 x float4:
//   [0] = (v0.x, v0.y, v0.z, proxy-hausdorff)   [1] = (v1.xyz, hausdorff)
//   [2] = (v2.xyz, 0)
constexpr int kTriF4 = 3;

// FP32 forward-error model for one voxel-pair distance: |d32 - d| <= kErrC * u * R,
// u = 2^-24, R = largest |coordinate| after translation to the pair's origin
// (the .w of the refine output).  kErrC is 8x the largest ratio measured
// against the FP64 oracle (tests/test_refine_gpu.py prints the measured ratio).
constexpr float kErrC = 64.0f;
constexpr float kUnitRoundoff = 5.9604645e-8f;

__host__ __device__ __forceinline__ float err_bound(float R) { return kErrC * kUnitRoundoff * R; }

struct Status {
    int code = 0;
    std::string msg;
};

}  // namespace tdp

#define TDP_CUDA_TRY(call)                                                                 \
    do {                                                                                   \
        cudaError_t _e = (call);                                                           \
        if (_e != cudaSuccess) {                                                           \
            return ::tdp::fail(ctx, TDP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
        }                                                                                  \
    } while (0)
