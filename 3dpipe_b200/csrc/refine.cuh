// refine.cuh -- launchers for the refine kernels (see refine.cu).  When
// n_items_dev is given, the kernel reads the exact item count from device
// memory and n_items is only an upper bound (it sizes the grid).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace tdp {

cudaError_t launch_refine_plain(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                float4* out, cudaStream_t s);
// tuned-kernel configurations (index 0 is the default); see refine.cu
constexpr int kTunedConfigs = 18;
struct TunedConfig {
    int chunk_a;      // A-side triangles staged per warp and chunk
    int ctas_per_sm;  // resident CTAs per SM the launch is sized for
};
TunedConfig tuned_config(int cfg);
cudaError_t launch_refine_tuned(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                                float4* out, unsigned* work_counter, unsigned long long* n_full, int num_sms,
                                int cfg, cudaStream_t s, const unsigned* n_items_dev = nullptr,
                                const float* init_bd = nullptr);
// init_bd (optional, per item): start the minimum distance at this bound and
// report x = FLT_MAX when no triangle pair lies below it; y and z (the
// Hausdorff minima) are then meaningless.  Used by the exact-distance stage.
// exact FP64 minimum distance per item (recheck of undecided object pairs)
// n_items is an upper bound when n_items_dev (the exact count, in device memory) is given
cudaError_t launch_refine_f64(const float4* triA, const float4* triB, const RefineItem* items, int n_items,
                              double* out, cudaStream_t s, const unsigned* n_items_dev = nullptr);
cudaError_t launch_pack_triangles(const float* data, const float* hd, size_t n, float4* tri, cudaStream_t s);

}  // namespace tdp
