// join_kernels.cu -- the filter and LOD-loop kernels of the spatial join.
//
// Reference correspondence (paths inside lyuheng/3dpipe):
//   k_pair_bounds      voxel_pair_dist_kernel_for_all_aggregate_distance and the
//                      min reduction of the streaming kernels
//                      (src/geometry/computing_gpu.cu:1984-2043, :2155-2359),
//                      voxel bounds voxel_dist_core (:1606-1631)
//   k_within_decide    filter-time classification (src/join/WithinJoin.cpp:164-252)
//                      and the per-LOD within decision (WithinJoin.cpp:769-792)
//   k_knn_rank         evaluate_knn_kernel (computing_gpu.cu:105-151) + the confirm
//                      cap in candidate order (src/join/KNNJoin.cpp:133-202), a
//                      warp per query with the cap taken by ballot
//   k_count/write_vps  record_valid_voxel_pairs_streaming_{knn,within}
//                      (computing_gpu.cu:2604-2812): voxel pairs with
//                      min <= object min-max (and <= tau for within), in (i,j) order
//   k_build_items      packing_data_stream's voxel-pair list (src/join/SpatialJoin.cpp:169-248),
//                      skipping voxels empty at this LOD (KNNJoin.cpp:1662)
//   k_apply_results    the per-voxel-pair bound update (KNNJoin.cpp:1668-1705)
//   k_pair_update      SpatialJoin::update_voxel_pair_list (SpatialJoin.cpp:48-69):
//                      object min over all voxel pairs, max over the updated ones,
//                      eviction of voxel pairs whose min exceeds that max
// The reference's block reductions in the filter assume a power-of-two block
// (computing_gpu.cu:2027-2033, blockDim = min(max_voxel_size, 1024)); the
// reductions here are exact for any voxel count.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <float.h>

#include "join_kernels.cuh"

namespace tdp {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ float wmin(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Squared box gap and squared core-core distance of two voxels (the terms of
// voxel_dist_core before its square roots).  Per axis the gap is
// max(0, alo - bhi, blo - ahi); for boxes with lo <= hi at most one of the two
// differences is positive, so this is the reference's branch
// (t2 < 0 ? t2^2 : t1 > 0 ? t1^2 : 0) with the same rounding.
__device__ __forceinline__ void vox_dist2(const float4 alo, const float4 ahi, const float4 ac, const float4 blo,
                                          const float4 bhi, const float4 bc, float& m, float& M) {
    const float gx = fmaxf(fmaxf(alo.x - bhi.x, blo.x - ahi.x), 0.f);
    const float gy = fmaxf(fmaxf(alo.y - bhi.y, blo.y - ahi.y), 0.f);
    const float gz = fmaxf(fmaxf(alo.z - bhi.z, blo.z - ahi.z), 0.f);
    const float dx = ac.x - bc.x, dy = ac.y - bc.y, dz = ac.z - bc.z;
    m = 0.f;
    M = 0.f;
    m += gx * gx;
    M += dx * dx;
    m += gy * gy;
    M += dy * dy;
    m += gz * gz;
    M += dz * dz;
}

// voxel_dist_core: box gap and core-core distance, a = tile-1 voxel, b = tile-2 voxel
__device__ __forceinline__ void vox_dist(const float4* __restrict__ va, const float4* __restrict__ vb, float& mn,
                                         float& mx) {
    float m, M;
    vox_dist2(va[0], va[1], va[2], vb[0], vb[1], vb[2], m, M);
    mn = sqrtf(m);
    mx = sqrtf(M);
}

// relative FP32 error of a box gap / core distance: a handful of roundings
constexpr float kVoxRel = 8.0f * kUnitRoundoff;

constexpr int kPBWarps = kBlock / 32;
constexpr int kPBCap = 64;    // tile-1 voxels staged per warp and pass
constexpr int kPBSmall = 24;  // below this many tile-2 voxels, lanes run over (a, b) pairs

// Object-pair bounds: min over voxel pairs of the box gap and of the core
// distance.  The square root is correctly rounded and so monotone:
// min_i sqrt(x_i) == sqrt(min_i x_i) exactly, so the minima are taken over the
// squared values and each object pair takes two square roots.  The query
// object's voxels are staged in shared memory (one warp per object pair).
__global__ void __launch_bounds__(kBlock) k_pair_bounds(JoinDev d) {
    __shared__ float4 sa[kPBWarps][kPBCap * 3];
    __shared__ float4 sb[kPBWarps][kPBSmall * 3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long vp = 0;  // voxel pairs seen by this warp (lane 0)
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        const int q = d.pq[p], t = d.pt[p];
        const uint32_t a0 = d.ovox1[q], a1 = d.ovox1[q + 1], b0 = d.ovox2[t], b1 = d.ovox2[t + 1];
        const int nb = (int)(b1 - b0);
        float m2 = FLT_MAX, M2 = FLT_MAX;
        bool early = false;  // reported before every voxel pair was seen
        const float etau = d.early_mixed ? (d.qk[q] == 0 ? d.qtau[q] : -1.f) : d.early_tau;
        if (nb < kPBSmall) {
            __syncwarp();
            for (int i = lane; i < nb * 3; i += 32) sb[w][i] = d.vox2[3 * (size_t)b0 + i];
        }
        for (uint32_t ac = a0; ac < a1 && !early; ac += kPBCap) {
            const int na = (int)min((uint32_t)kPBCap, a1 - ac);
            __syncwarp();
            for (int i = lane; i < na * 3; i += 32) sa[w][i] = d.vox1[3 * (size_t)ac + i];
            __syncwarp();
            if (nb >= kPBSmall) {
                // two tile-2 voxels per lane share every staged tile-1 voxel; a
                // missing second one repeats the first (harmless for a minimum)
                for (int bb = 0; bb < nb && !early; bb += 64) {
                    const int b = bb + lane;
                    if (b < nb) {
                        const float4* v0 = d.vox2 + 3 * ((size_t)b0 + b);
                        const float4* v1 = b + 32 < nb ? v0 + 96 : v0;
                        const float4 lo0 = __ldg(v0), hi0 = __ldg(v0 + 1), c0 = __ldg(v0 + 2);
                        const float4 lo1 = __ldg(v1), hi1 = __ldg(v1 + 1), c1 = __ldg(v1 + 2);
                        for (int i = 0; i < na; ++i) {
                            const float4 alo = sa[w][3 * i], ahi = sa[w][3 * i + 1], acr = sa[w][3 * i + 2];
                            float m, M, m1, M1;
                            vox_dist2(alo, ahi, acr, lo0, hi0, c0, m, M);
                            vox_dist2(alo, ahi, acr, lo1, hi1, c1, m1, M1);
                            m2 = fminf(m2, fminf(m, m1));
                            M2 = fminf(M2, fminf(M, M1));
                        }
                    }
                    if (etau >= 0.f) {
                        // a core distance is a distance between two surface points,
                        // so it bounds the pair's distance from above: the tuned
                        // within decision (max + error band <= tau) is final
                        const float mx = sqrtf(M2);
                        early = __any_sync(0xffffffffu, mx + kVoxRel * mx <= etau);
                    }
                }
            } else if (nb > 0) {
                const int n = na * nb;
                int i = lane / nb, b = lane - i * nb;
                for (int k = lane; k < n; k += 32) {
                    float m, M;
                    vox_dist2(sa[w][3 * i], sa[w][3 * i + 1], sa[w][3 * i + 2], sb[w][3 * b], sb[w][3 * b + 1],
                              sb[w][3 * b + 2], m, M);
                    m2 = fminf(m2, m);
                    M2 = fminf(M2, M);
                    b += 32;
                    while (b >= nb) { b -= nb; ++i; }
                }
            }
        }
        m2 = wmin(m2);
        M2 = wmin(M2);
        if (early) {
            if (lane == 0) {
                const float mx = sqrtf(M2);
                d.pmn[p] = 0.f;  // not computed: the pair is decided
                d.pmx[p] = mx;
                d.perr[p] = kVoxRel * mx;
                d.pstat[p] = kReported;
                vp += (unsigned long long)(a1 - a0) * (b1 - b0);
            }
            continue;
        }
        if (lane == 0) {
            const float mn = m2 == FLT_MAX ? FLT_MAX : sqrtf(m2);
            const float mx = M2 == FLT_MAX ? FLT_MAX : sqrtf(M2);
            d.pmn[p] = mn;
            d.pmx[p] = mx;
            d.perr[p] = kVoxRel * fmaxf(mn, mx);
            d.pstat[p] = kUndecided;
            vp += (unsigned long long)(a1 - a0) * (b1 - b0);
        }
    }
    if (lane == 0 && vp && d.stat_vp) atomicAdd(d.stat_vp, vp);
}

__global__ void k_within_decide(JoinDev d, float tau_all, int tuned) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.P; p += gridDim.x * blockDim.x) {
        if (d.pstat[p] != kUndecided) continue;
        float tau = tau_all;
        if (d.qk) {
            const int q = d.pq[p];
            if (d.qk[q] > 0) continue;  // a kNN object of a mixed batch
            tau = d.qtau[q];
        }
        const float e = tuned ? d.perr[p] : 0.f;
        if (d.pmx[p] + e <= tau) d.pstat[p] = kReported;
        else if (d.pmn[p] - e > tau) d.pstat[p] = kDropped;
    }
}

// One warp per query object.  Pass 1: each lane takes candidates lane,
// lane + 32, ... and applies the bulk rule against every other undecided
// candidate (CONFIRMED if fewer than K - confirmed candidates may be closer,
// REMOVED if at least that many are surely closer).  Pass 2: the cap in
// candidate order, 32 candidates at a time: a candidate is acted on while the
// confirmations before it (a ballot and a prefix count) leave an open slot,
// which is what the reference's sequential loop does (it stops at the first
// candidate that finds the K slots full).
__global__ void __launch_bounds__(kBlock) k_knn_rank(JoinDev d, int K_all, int tuned, int* __restrict__ st) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < d.N1; q += nw) {
        const int K = d.qk ? d.qk[q] : K_all;
        if (K <= 0) continue;  // a within object of a mixed batch (warp-uniform)
        const int64_t b = d.qoff[q], e = d.qoff[q + 1];
        int conf = d.qconf[q];
        if (conf < K) {
            const int cand_left = K - conf;
            for (int64_t i = b + lane; i < e; i += 32) {
                if (d.pstat[i] != kUndecided) continue;
                const float ei = tuned ? d.perr[i] : 0.f;
                const float lo = d.pmn[i] - ei, hi = d.pmx[i] + ei;
                int sure = 0, maybe = 0;
                for (int64_t j = b; j < e; ++j) {
                    if (j == i || d.pstat[j] != kUndecided) continue;
                    const float ej = tuned ? d.perr[j] : 0.f;
                    if (lo >= d.pmx[j] + ej) ++sure;
                    if (!(hi <= d.pmn[j] - ej)) ++maybe;
                }
                st[i] = maybe < cand_left ? 1 : (sure >= cand_left ? 2 : 0);
            }
            __syncwarp();
            for (int64_t base = b; base < e && conf < K; base += 32) {
                const int64_t i = base + lane;
                const bool und = i < e && d.pstat[i] == kUndecided;
                const int s = und ? st[i] : 0;
                const unsigned cm = __ballot_sync(0xffffffffu, s == 1);
                if (und && conf + __popc(cm & lt) < K) {
                    if (s == 1) d.pstat[i] = kReported;
                    else if (s == 2) d.pstat[i] = kDropped;
                }
                conf = min(K, conf + __popc(cm));
            }
            if (lane == 0) d.qconf[q] = conf;
        }
        if (conf >= K)  // query complete: nothing left to refine for it
            for (int64_t i = b + lane; i < e; i += 32)
                if (d.pstat[i] == kUndecided) d.pstat[i] = kDropped;
        __syncwarp();
    }
}

template <bool WRITE>
__global__ void __launch_bounds__(kBlock) k_vps(JoinDev d, int within_all, float tau_all, int tuned,
                                                 int64_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        if (d.pstat[p] != kUndecided) {
            if (!WRITE && lane == 0) cnt[p] = 0;
            continue;
        }
        const int q = d.pq[p], t = d.pt[p];
        const int within = d.qk ? d.qk[q] == 0 : within_all;
        const float tau = d.qk ? d.qtau[q] : tau_all;
        const uint32_t a0 = d.ovox1[q], b0 = d.ovox2[t];
        const uint32_t n1 = d.ovox1[q + 1] - a0, n2 = d.ovox2[t + 1] - b0;
        const float slack = tuned ? d.perr[p] : 0.f;
        const float lim = d.pmx[p] + slack;
        const uint64_t total = (uint64_t)n1 * n2;
        int64_t pos = WRITE ? d.pvp[p] : 0;
        int64_t count = 0;
        for (uint64_t base = 0; base < total; base += 32) {
            const uint64_t k = base + lane;
            bool keep = false;
            float m = 0.f, M = 0.f;
            uint32_t a = 0, bb = 0;
            if (k < total) {
                a = (uint32_t)(k / n2);
                bb = (uint32_t)(k - (uint64_t)a * n2);
                const float4* va = d.vox1 + 3 * (size_t)(a0 + a);
                const float4* vb = d.vox2 + 3 * (size_t)(b0 + bb);
                vox_dist(va, vb, m, M);
                if (d.isect) {
                    // aab::intersect: strict overlap on every axis
                    const float4 alo = va[0], ahi = va[1], blo = vb[0], bhi = vb[1];
                    keep = !(blo.x >= ahi.x || bhi.x <= alo.x || blo.y >= ahi.y || bhi.y <= alo.y ||
                             blo.z >= ahi.z || bhi.z <= alo.z);
                } else {
                    keep = (m - slack <= lim) && (!within || m - slack <= tau);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (WRITE && keep) {
                const int64_t w = pos + __popc(bal & ((1u << lane) - 1u));
                d.vpa[w] = (int)(a0 + a);
                d.vpb[w] = (int)(b0 + bb);
                d.vpair[w] = p;
                d.vmn[w] = m;
                d.vmx[w] = M;
                d.verr[w] = kVoxRel * fmaxf(m, M);
                d.valive[w] = 1;
                d.vupd[w] = -1;
            }
            pos += __popc(bal);
            count += __popc(bal);
        }
        if (!WRITE && lane == 0) cnt[p] = count;
    }
}

// One slot claim and one triangle-pair sum per warp: lane 0 adds the warp's
// item count and n1*n2 sum to the counters, the lanes write at the claimed
// base plus their rank among the warp's items.  (The items form a set: their
// order never changes a result.)
// The preset of a within item at the last LOD (LOD 100): its query's
// distance plus twice the largest FP32 error of a triangle pair that could
// be within it.  Such a pair's coordinates, taken from a vertex of the A
// voxel, stay below tau + both voxel extents (R), so its FP32 distance is
// below tau + err_bound(R): an item with nothing below the preset has no
// pair within tau.  kNN items get FLT_MAX (no preset).
__device__ __forceinline__ float within_preset(const JoinDev& d, int p, int a, int b, float tau_all) {
    float tau = tau_all;
    if (d.qk) {
        const int q = d.pq[p];
        if (d.qk[q] > 0) return FLT_MAX;
        tau = d.qtau[q];
    }
    const float4* va = d.vox1 + 3 * (size_t)a;
    const float4* vb = d.vox2 + 3 * (size_t)b;
    const float4 alo = va[0], ahi = va[1], blo = vb[0], bhi = vb[1];
    const float da = (ahi.x - alo.x) + (ahi.y - alo.y) + (ahi.z - alo.z);
    const float db = (bhi.x - blo.x) + (bhi.y - blo.y) + (bhi.z - blo.z);
    const float R = (tau + da + db) * 1.001f + 1.f;
    return tau + 2.f * err_bound(R) + 1e-6f;
}

// preset != NULL (the tuned form's last LOD of a join with within queries):
// also write each item's preset (within_preset)
__global__ void k_build_items(JoinDev d, const uint32_t* __restrict__ vt1, const uint32_t* __restrict__ vt2,
                              RefineItem* __restrict__ items, int* __restrict__ item_vp, unsigned* __restrict__ counter,
                              float* __restrict__ preset, float tau_all) {
    // counter[0] = items, counter[2..3] = sum n1*n2 (u64)
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations (the bound is rounded up to whole warps)
    const int64_t vend = (d.V + 31) & ~(int64_t)31;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < vend; v += stride) {
        bool ok = v < d.V && d.valive[v] && d.pstat[d.vpair[v]] == kUndecided;
        uint32_t o1 = 0, n1 = 0, o2 = 0, n2 = 0;
        int a = 0, b = 0;
        if (ok) {
            a = d.vpa[v];
            b = d.vpb[v];
            o1 = vt1[a]; n1 = vt1[a + 1] - o1;
            o2 = vt2[b]; n2 = vt2[b + 1] - o2;
            ok = n1 > 0 && n2 > 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (!m) continue;
        unsigned long long tp = ok ? (unsigned long long)n1 * n2 : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tp += __shfl_xor_sync(0xffffffffu, tp, o);
        unsigned base = 0;
        if (lane == 0) {
            base = atomicAdd(counter, (unsigned)__popc(m));
            atomicAdd(reinterpret_cast<unsigned long long*>(counter + 2), tp);
        }
        base = __shfl_sync(0xffffffffu, base, 0);
        if (ok) {
            const unsigned w = base + __popc(m & ((1u << lane) - 1u));
            items[w] = RefineItem{o1, n1, o2, n2};
            item_vp[w] = (int)v;
            if (preset) preset[w] = within_preset(d, d.vpair[v], a, b, tau_all);
        }
    }
}

// A voxel pair whose refine found nothing below its preset is out of its
// query's reach: both its bounds go to kFar, so it never lowers the pair's
// minimum, never reports it, and adds no error term.
constexpr float kFar = 3.0e38f;

__global__ void k_apply_results(JoinDev d, const float4* __restrict__ res, const int* __restrict__ item_vp, int W_host,
                                const unsigned* W_dev, int highest, int level, int li, int stamp,
                                const float* __restrict__ preset) {
    const int W = W_dev ? (int)*W_dev : W_host;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        const int v = item_vp[w];
        const float4 r = res[w];
        float mn = d.vmn[v], mx = d.vmx[v];
        const float e = err_bound(r.w);
        if (highest && preset) {
            const float pb = preset[w];
            if (pb < FLT_MAX && !(r.x < pb)) {
                d.vmn[v] = kFar;
                d.vmx[v] = kFar;
                d.verr[v] = fmaxf(d.verr[v], e);
                d.vupd[v] = stamp;
                continue;
            }
        }
        if (highest) {
            mn = r.x;
            mx = r.x;
        } else if (level == 2) {
            mn = fminf(mn, r.y);
            mx = fminf(mx, r.z);
        } else if (level == 1) {
            const int p = d.vpair[v];
            const int q = d.pq[p], t = d.pt[p];
            mn = fminf(mn, r.x - d.ohd1[q * 5 + li] - d.ohd2[t * 5 + li]);
            mx = fminf(mx, r.x + d.ophd1[q * 5 + li] + d.ophd2[t * 5 + li]);
        } else {
            mx = fminf(mx, r.x);
        }
        d.vmn[v] = mn;
        d.vmx[v] = mx;
        d.verr[v] = fmaxf(d.verr[v], e + 4.f * kUnitRoundoff * fmaxf(fabsf(mn), fabsf(mx)));
        d.vupd[v] = stamp;
    }
}

// ---- FP64 recheck (tuned form) of pairs still undecided after the last LOD ----
__global__ void k_recheck_items(JoinDev d, const uint32_t* __restrict__ vt1, const uint32_t* __restrict__ vt2,
                                RefineItem* __restrict__ items, int* __restrict__ item_vp, double* __restrict__ vexact,
                                unsigned* __restrict__ counter) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < d.V; v += (int64_t)gridDim.x * blockDim.x) {
        if (!d.valive[v] || d.pstat[d.vpair[v]] != kUndecided) continue;
        vexact[v] = 1e300;
        const int a = d.vpa[v], b = d.vpb[v];
        const uint32_t o1 = vt1[a], n1 = vt1[a + 1] - o1, o2 = vt2[b], n2 = vt2[b + 1] - o2;
        if (!n1 || !n2) continue;
        const unsigned w = atomicAdd(counter, 1u);
        items[w] = RefineItem{o1, n1, o2, n2};
        item_vp[w] = (int)v;
    }
}

__global__ void k_recheck_apply(const double* __restrict__ res, const int* __restrict__ item_vp, int W_host,
                                const unsigned* W_dev, double* __restrict__ vexact) {
    const int W = W_dev ? (int)*W_dev : W_host;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) vexact[item_vp[w]] = res[w];
}

__global__ void __launch_bounds__(kBlock) k_recheck_pairs(JoinDev d, const double* __restrict__ vexact,
                                                          double* __restrict__ pexact, int within_all,
                                                          float tau_all) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        if (d.pstat[p] != kUndecided) continue;
        double D = 1e300;
        for (int64_t v = d.pvp[p] + lane; v < d.pvp[p + 1]; v += 32)
            if (d.valive[v]) D = vexact[v] < D ? vexact[v] : D;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double x = __shfl_xor_sync(0xffffffffu, D, o);
            D = x < D ? x : D;
        }
        if (lane == 0) {
            const int q = d.pq[p];
            const int within = d.qk ? d.qk[q] == 0 : within_all;
            const float tau = d.qk ? d.qtau[q] : tau_all;
            pexact[p] = D;
            d.pmn[p] = d.pmx[p] = (float)D;
            if (within) d.pstat[p] = D <= (double)tau ? kReported : kDropped;
        }
    }
}

// kNN: the still-undecided candidates of a query compete for its open slots by exact distance
__global__ void k_recheck_knn(JoinDev d, int K_all, const double* __restrict__ pexact) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < d.N1; q += gridDim.x * blockDim.x) {
        const int K = d.qk ? d.qk[q] : K_all;
        if (K <= 0) continue;
        const int64_t b = d.qoff[q], e = d.qoff[q + 1];
        int conf = d.qconf[q];
        while (conf < K) {
            int64_t best = -1;
            for (int64_t i = b; i < e; ++i)
                if (d.pstat[i] == kUndecided && (best < 0 || pexact[i] < pexact[best])) best = i;
            if (best < 0) break;
            d.pstat[best] = kReported;
            ++conf;
        }
        for (int64_t i = b; i < e; ++i)
            if (d.pstat[i] == kUndecided) d.pstat[i] = kDropped;
        d.qconf[q] = conf;
    }
}

// decide != 0: the within decision of k_within_decide is taken here too, for
// the within query objects, as soon as the pair's bounds are known (the tuned
// LOD loop; it saves a launch and a pass over the pairs per LOD)
__global__ void __launch_bounds__(kBlock) k_pair_update(JoinDev d, int stamp, int tuned, int decide, float tau_all) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < d.P; p += nw) {
        if (d.pstat[p] != kUndecided) continue;
        const int64_t b = d.pvp[p], e = d.pvp[p + 1];
        float minmax = INFINITY, mindist = FLT_MAX, err = 0.f;
        for (int64_t v = b + lane; v < e; v += 32) {
            if (!d.valive[v]) continue;
            mindist = fminf(mindist, d.vmn[v]);
            err = fmaxf(err, d.verr[v]);
            if (d.vupd[v] == stamp) minmax = fminf(minmax, d.vmx[v]);
        }
        minmax = wmin(minmax);
        mindist = wmin(mindist);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) err = fmaxf(err, __shfl_xor_sync(0xffffffffu, err, o));
        // evict voxel pairs that cannot hold the minimum; the tuned form keeps any
        // whose FP32 bounds overlap within the error band
        const float slack = tuned ? 2.f * err : 0.f;
        for (int64_t v = b + lane; v < e; v += 32)
            if (d.valive[v] && d.vmn[v] - slack > minmax) d.valive[v] = 0;
        if (lane == 0) {
            d.pmn[p] = mindist;
            d.pmx[p] = minmax;
            d.perr[p] = err;
            if (decide) {  // as k_within_decide
                float tau = tau_all;
                bool within = true;
                if (d.qk) {
                    const int q = d.pq[p];
                    within = d.qk[q] <= 0;
                    tau = d.qtau[q];
                }
                if (within) {
                    const float e = tuned ? err : 0.f;
                    if (minmax + e <= tau) d.pstat[p] = kReported;
                    else if (mindist - e > tau) d.pstat[p] = kDropped;
                }
            }
        }
    }
}

__global__ void k_count_status(JoinDev d, unsigned* __restrict__ c) {
    unsigned und = 0, rep = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.P; p += gridDim.x * blockDim.x) {
        und += d.pstat[p] == kUndecided;
        rep += d.pstat[p] == kReported;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        und += __shfl_xor_sync(0xffffffffu, und, o);
        rep += __shfl_xor_sync(0xffffffffu, rep, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (und) atomicAdd(c + 0, und);
        if (rep) atomicAdd(c + 1, rep);
    }
}

// Result keys: query * n2 + result id for reported pairs, `none` (= n1 * n2)
// for the rest, so one radix sort over every pair puts the reported ones
// first, ordered by (query, result id); the payload is the pair index.
__global__ void k_collect_keys(JoinDev d, long long n2, unsigned long long none, unsigned long long* __restrict__ keys,
                               int* __restrict__ vals, unsigned* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < d.P; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = base + threadIdx.x;
        const bool rep = p < d.P && d.pstat[p] == kReported;
        if (p < d.P) {
            keys[p] = rep ? (unsigned long long)d.pq[p] * (unsigned long long)n2 + (unsigned)d.pt[p] : none;
            vals[p] = (int)p;
        }
        const unsigned m = __ballot_sync(0xffffffffu, rep);
        if (lane == 0 && m) atomicAdd(counter, (unsigned)__popc(m));
    }
}

__global__ void k_split(JoinDev d, const unsigned long long* __restrict__ keys, const int* __restrict__ vals,
                        long long n2, unsigned long long none, const double* __restrict__ pexact,
                        int* __restrict__ oq, int* __restrict__ ot, float* __restrict__ od, double* __restrict__ od64) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.P; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k == none) break;  // sorted: every later key is `none` too
        const int p = vals[i];
        oq[i] = (int)(k / (unsigned long long)n2);
        ot[i] = (int)(k % (unsigned long long)n2);
        od[i] = d.pmx[p];
        if (od64) od64[i] = pexact ? pexact[p] : (double)d.pmx[p];
    }
}

int grid_for(int64_t n, int per_block, int cap = 148 * 32) {
    int64_t g = (n + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

}  // namespace

cudaError_t launch_pair_bounds(const JoinDev& d, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    k_pair_bounds<<<grid_for(d.P, kBlock / 32), kBlock, 0, s>>>(d);
    return cudaGetLastError();
}
cudaError_t launch_within_decide(const JoinDev& d, float tau, int tuned, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    k_within_decide<<<grid_for(d.P, 256), 256, 0, s>>>(d, tau, tuned);
    return cudaGetLastError();
}
cudaError_t launch_knn_rank(const JoinDev& d, int K, int tuned, int* st, cudaStream_t s) {
    if (d.N1 <= 0) return cudaSuccess;
    k_knn_rank<<<grid_for(d.N1, kBlock / 32, 148 * 32), kBlock, 0, s>>>(d, K, tuned, st);
    return cudaGetLastError();
}
cudaError_t launch_count_vps(const JoinDev& d, int within, float tau, int tuned, int64_t* cnt, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    k_vps<false><<<grid_for(d.P, kBlock / 32), kBlock, 0, s>>>(d, within, tau, tuned, cnt);
    return cudaGetLastError();
}
cudaError_t launch_write_vps(const JoinDev& d, int within, float tau, int tuned, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    k_vps<true><<<grid_for(d.P, kBlock / 32), kBlock, 0, s>>>(d, within, tau, tuned, nullptr);
    return cudaGetLastError();
}
cudaError_t launch_build_items(const JoinDev& d, const uint32_t* vt1, const uint32_t* vt2, RefineItem* items,
                               int* item_vp, unsigned* counter, cudaStream_t s, float* preset, float tau) {
    if (d.V <= 0) return cudaSuccess;
    k_build_items<<<grid_for(d.V, 256), 256, 0, s>>>(d, vt1, vt2, items, item_vp, counter, preset, tau);
    return cudaGetLastError();
}
cudaError_t launch_apply_results(const JoinDev& d, const float4* res, const int* item_vp, int W, int highest,
                                 int level, int li, int stamp, cudaStream_t s, const unsigned* W_dev,
                                 const float* preset) {
    if (W <= 0) return cudaSuccess;
    k_apply_results<<<grid_for(W, 256), 256, 0, s>>>(d, res, item_vp, W, W_dev, highest, level, li, stamp, preset);
    return cudaGetLastError();
}
cudaError_t launch_pair_update(const JoinDev& d, int stamp, int tuned, cudaStream_t s, int decide, float tau) {
    if (d.P <= 0) return cudaSuccess;
    k_pair_update<<<grid_for(d.P, kBlock / 32), kBlock, 0, s>>>(d, stamp, tuned, decide, tau);
    return cudaGetLastError();
}
cudaError_t launch_recheck_items(const JoinDev& d, const uint32_t* vt1, const uint32_t* vt2, RefineItem* items,
                                 int* item_vp, double* vexact, unsigned* counter, cudaStream_t s) {
    if (d.V <= 0) return cudaSuccess;
    k_recheck_items<<<grid_for(d.V, 256), 256, 0, s>>>(d, vt1, vt2, items, item_vp, vexact, counter);
    return cudaGetLastError();
}
cudaError_t launch_recheck_finish(const JoinDev& d, const double* res, const int* item_vp, int W, double* vexact,
                                  double* pexact, int knn, int K, float tau, cudaStream_t s, const unsigned* W_dev) {
    if (W > 0) k_recheck_apply<<<grid_for(W, 256), 256, 0, s>>>(res, item_vp, W, W_dev, vexact);
    if (d.P > 0) k_recheck_pairs<<<grid_for(d.P, kBlock / 32), kBlock, 0, s>>>(d, vexact, pexact, !knn, tau);
    if ((knn || d.qk) && d.N1 > 0) k_recheck_knn<<<grid_for(d.N1, 128), 128, 0, s>>>(d, K, pexact);
    return cudaGetLastError();
}
cudaError_t launch_count_status(const JoinDev& d, unsigned* c, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    k_count_status<<<grid_for(d.P, 256, 148 * 8), 256, 0, s>>>(d, c);
    return cudaGetLastError();
}
static int key_bits(unsigned long long none) {
    int b = 1;
    while (b < 64 && (none >> b)) ++b;
    return b;
}
cudaError_t collect_sort_bytes(int64_t P, long long n1, long long n2, size_t& bytes) {
    bytes = 0;
    if (P <= 0) return cudaSuccess;
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
    cub::DoubleBuffer<int> v(nullptr, nullptr);
    return cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, (int)P, 0,
                                           key_bits((unsigned long long)n1 * (unsigned long long)n2));
}
cudaError_t launch_collect(const JoinDev& d, long long n2, unsigned long long* keys[2], int* vals[2], void* temp,
                           size_t temp_bytes, unsigned* counter, const double* pexact, int* oq, int* ot, float* od,
                           double* od64, cudaStream_t s) {
    if (d.P <= 0) return cudaSuccess;
    const unsigned long long none = (unsigned long long)d.N1 * (unsigned long long)n2;
    k_collect_keys<<<grid_for(d.P, 256), 256, 0, s>>>(d, n2, none, keys[0], vals[0], counter);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cub::DoubleBuffer<unsigned long long> k(keys[0], keys[1]);
    cub::DoubleBuffer<int> v(vals[0], vals[1]);
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k, v, (int)d.P, 0, key_bits(none), s);
    if (e != cudaSuccess) return e;
    k_split<<<grid_for(d.P, 256), 256, 0, s>>>(d, k.Current(), v.Current(), n2, none, pexact, oq, ot, od, od64);
    return cudaGetLastError();
}

cudaError_t scan_counts(const int64_t* cnt, int64_t* out, int n, void* temp, size_t& temp_bytes, cudaStream_t s) {
    // exclusive scan of n+1 values (cnt[n] must be 0) so out[n] is the total
    return cub::DeviceScan::ExclusiveSum(temp, temp_bytes, cnt, out, n + 1, s);
}

}  // namespace tdp
