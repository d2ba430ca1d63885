// cand_kernels.cuh -- object candidate generation on the GPU (the first filter level).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ctx.cuh"
#include "storage/dev_tile.h"

namespace tdp {

// Candidates of every tile-1 object against tile 2, the same set and order as
// generate_candidates() (src/index/candidates.cpp) and the reference octree.
// On success pq/pt (object pairs, grouped by query object) and qoff ([n1+1]
// CSR) are device buffers owned by the context's scratch, P is the pair count.
// n_redone: kNN queries whose ring search brought more points than a warp's
// shared-memory buffer holds; they are redone on the device with a global
// buffer that cannot overflow, so the result is always complete.
// qk / qtau (device, optional): per tile-1 object K (> 0, kNN) or 0 (within,
// distance qtau); NULL: every object uses (knn, K, tau).
// Only tile-1 objects [q_begin, q_end) get candidates (q_end < 0: all).
int device_candidates(tdp_ctx* ctx, const tdp_tile* t1, const tdp_tile* t2, bool self, bool knn, int K, float tau,
                      Buf& pq_buf, Buf& pt_buf, Buf& qoff_buf, long& P, long& n_redone, const int* qk = nullptr,
                      const float* qtau = nullptr, bool isect = false, long q_begin = 0, long q_end = -1);

}  // namespace tdp
