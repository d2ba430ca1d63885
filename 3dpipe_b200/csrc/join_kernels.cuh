// join_kernels.cuh -- device state of one join and the launchers of its kernels.
// The orchestration (LOD loop, decisions, result collection) lives in
// src/join/join_driver.cpp; every kernel here is one step of the reference's
// filter + LOD refine loop (reference src/join/KNNJoin.cpp, WithinJoin.cpp,
// src/geometry/computing_gpu.cu), restated for device-resident state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tdp {

enum PairStatus : uint8_t { kUndecided = 0, kReported = 1, kDropped = 2 };

struct JoinDev {
    // tiles
    const float4* vox1;
    const uint32_t* ovox1;
    const float4* vox2;
    const uint32_t* ovox2;
    const float* ohd1;
    const float* ophd1;
    const float* ohd2;
    const float* ophd2;
    // object pairs (candidates), grouped by query object
    int P;
    const int* pq;
    const int* pt;
    float* pmn;
    float* pmx;
    float* perr;  // FP32 error bound of the pair range (tuned form)
    uint8_t* pstat;
    int64_t* pvp;  // [P+1] first voxel pair of each pair
    // queries
    int N1;
    const int64_t* qoff;  // [N1+1]
    int* qconf;
    // per query object query (a batch of different requests), or NULL when
    // every object uses the call's scalar query: qk[q] = K (> 0, kNN) or 0
    // (within, distance qtau[q])
    const int* qk;
    const float* qtau;
    // intersect query: voxel pairs are kept when their boxes overlap strictly
    int isect;
    // tuned form: the filter reports a within pair as soon as one voxel pair's
    // core distance (plus its error band) is within its distance -- early_tau
    // for a single within query (< 0: off), qtau[q] of within objects when
    // early_mixed is set
    float early_tau;
    int early_mixed;
    // voxel pairs kept after the filter
    int64_t V;
    int* vpa;
    int* vpb;
    int* vpair;
    float* vmn;
    float* vmx;
    float* verr;
    uint8_t* valive;
    int* vupd;
    unsigned long long* stat_vp;  // voxel pairs evaluated by the filter (statistic)
};

// filter: per object pair, min box gap and min core distance over all voxel pairs
cudaError_t launch_pair_bounds(const JoinDev& d, cudaStream_t s);
// within: classify pairs at the filter (min > tau drop, max <= tau report)
cudaError_t launch_within_decide(const JoinDev& d, float tau, int tuned, cudaStream_t s);
// kNN: the bulk rank rule per query object, then the confirm cap at K
cudaError_t launch_knn_rank(const JoinDev& d, int K, int tuned, int* scratch_status, cudaStream_t s);
// voxel-pair compaction of undecided pairs: count, then write in order
cudaError_t launch_count_vps(const JoinDev& d, int within, float tau, int tuned, int64_t* cnt, cudaStream_t s);
cudaError_t launch_write_vps(const JoinDev& d, int within, float tau, int tuned, cudaStream_t s);
// LOD step
// preset != NULL: also each item's preset for the refine's init_bd (the
// tuned form's last LOD, LOD 100, of a join with within queries): the
// query's distance plus the FP32 error band, FLT_MAX for kNN items
cudaError_t launch_build_items(const JoinDev& d, const uint32_t* vtri1, const uint32_t* vtri2, RefineItem* items,
                               int* item_vp, unsigned* counter, cudaStream_t s, float* preset = nullptr,
                               float tau = 0.f);
// W: item count, or an upper bound when W_dev (the exact count in device memory) is given;
// preset: the presets the last LOD's refine ran with (NULL: none)
cudaError_t launch_apply_results(const JoinDev& d, const float4* res, const int* item_vp, int W, int highest,
                                 int level, int lod_idx, int stamp, cudaStream_t s, const unsigned* W_dev = nullptr,
                                 const float* preset = nullptr);
// decide != 0 also takes the within decision (k_within_decide) of each pair
cudaError_t launch_pair_update(const JoinDev& d, int stamp, int tuned, cudaStream_t s, int decide = 0, float tau = 0.f);
// tuned form: FP64 recheck of the pairs left undecided after LOD 100
cudaError_t launch_recheck_items(const JoinDev& d, const uint32_t* vtri1, const uint32_t* vtri2, RefineItem* items,
                                 int* item_vp, double* vexact, unsigned* counter, cudaStream_t s);
cudaError_t launch_recheck_finish(const JoinDev& d, const double* res, const int* item_vp, int W, double* vexact,
                                  double* pexact, int knn, int K, float tau, cudaStream_t s,
                                  const unsigned* W_dev = nullptr);
cudaError_t launch_count_status(const JoinDev& d, unsigned* counters, cudaStream_t s);
// Reported pairs as (query, result id, distance) rows sorted by (query,
// result id) on the device: the first *counter rows of out_q/out_t/out_d
// (out_d = the pair's upper bound pmx; out_d64, if not NULL, = pexact when
// given, else pmx widened).  keys[0..1] / vals[0..1] are P-element double
// buffers for the radix sort, temp its workspace of collect_sort_bytes()
// bytes; n2 is the tile-2 object count.
cudaError_t collect_sort_bytes(int64_t P, long long n1, long long n2, size_t& bytes);
cudaError_t launch_collect(const JoinDev& d, long long n2, unsigned long long* keys[2], int* vals[2], void* temp,
                           size_t temp_bytes, unsigned* counter, const double* pexact, int* out_q, int* out_t,
                           float* out_d, double* out_d64, cudaStream_t s);
// exclusive scan of n int64 counts into out[0..n] (out[n] = total)
cudaError_t scan_counts(const int64_t* cnt, int64_t* out, int n, void* temp, size_t& temp_bytes, cudaStream_t s);

}  // namespace tdp
