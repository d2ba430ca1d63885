/*
 * tdp.h -- C ABI of the B200 (sm_100a) spatial-join hot path: the multi-level
 * filter and the LOD refine of 3DPipe's `tdbase join -q nn|within`.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (TDP_OK == 0); on failure tdp_last_error(ctx) describes the cause.  Nothing
 * here calls exit() or aborts.  A context owns all device memory it allocates;
 * the caller owns every host buffer it passes in or out.  One context must not
 * be used from two threads at the same time; separate contexts may.
 *
 * Reference interfaces replaced (paths inside lyuheng/3dpipe):
 *   tdp_ctx_create / tdp_ctx_destroy   geometry_computer::init_gpus + initialize_refine_stream
 *                                      (src/geometry/geometry_computer.cpp:78-84,
 *                                       src/geometry/computing_gpu.cu:36-43)
 *   tdp_tile_upload                    Tile::load + HiMesh_Wrapper(RAW) + allocateVoxelsForAll
 *                                      (src/storage/tile_IO.cpp:13-49,
 *                                       src/spatial/himesh_wrapper.cpp:17-83,
 *                                       src/geometry/computing_gpu.cu:1708-1772)
 *   tdp_join                           SpatialJoin::nearest_neighbor_chunking / within_chunking
 *                                      (src/join/KNNJoin.cpp:1524-1811,
 *                                       src/join/WithinJoin.cpp:644-813)
 *   tdp_refine_batch                   geometry_computer::get_distance_gpu[_stream] ->
 *                                      MeshDist_batch_gpu_op_shm_flat_stream
 *                                      (src/geometry/geometry_computer.cpp:86-151,
 *                                       src/geometry/computing_gpu.cu:6540-6658)
 */
#ifndef TDP_H
#define TDP_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define TDP_OK 0
#define TDP_ERR_ARG 1     /* bad argument (null pointer, size out of range)      */
#define TDP_ERR_CUDA 2    /* a CUDA runtime call failed                          */
#define TDP_ERR_NOMEM 3   /* device memory budget exceeded / allocation failed   */
#define TDP_ERR_FORMAT 4  /* malformed RAW .dt tile bytes                        */
#define TDP_ERR_TIMEOUT 5 /* a bounded device-side wait ran out                  */
#define TDP_ERR_STATE 6   /* call not valid in the current state                 */
#define TDP_ERR_NODEV 7   /* no CUDA device / not an sm_100 device               */

typedef struct tdp_ctx tdp_ctx;
typedef struct tdp_tile tdp_tile;
typedef struct tdp_result tdp_result;

/* ---- context --------------------------------------------------------------
 * device: CUDA ordinal.  budget_bytes: cap on device memory this context may
 * hold (0 = no cap beyond what the device has).  flags: reserved, pass 0. */
int tdp_ctx_create(int device, size_t budget_bytes, unsigned flags, tdp_ctx **out);
int tdp_ctx_destroy(tdp_ctx *ctx);
const char *tdp_last_error(const tdp_ctx *ctx);
/* device memory currently held by the context, and its high-water mark */
int tdp_ctx_memory(const tdp_ctx *ctx, size_t *in_use, size_t *peak);

/* statistics of the last tdp_refine_batch / tdp_join call on this context;
 * times are device times taken with CUDA events on the context's stream */
typedef struct {
    double refine_ms;                /* refine kernels                          */
    double filter_ms;                /* filter kernels                          */
    double total_ms;                 /* the whole call                          */
    unsigned long long full_evals;   /* triangle pairs fully evaluated          */
    double tri_pairs;                /* sum of n1*n2 over refined voxel pairs   */
    long refine_items;               /* voxel pairs refined, all LODs           */
    long refine_launches;            /* refine kernel launches                  */
    long recheck_pairs;              /* object pairs recomputed in FP64         */
    long filter_pairs;               /* object pairs through the filter         */
    double filter_voxel_pairs;       /* voxel pairs evaluated by the filter     */
    long kernel_launches;            /* all kernels launched by the call        */
} tdp_stats;
int tdp_last_stats(const tdp_ctx *ctx, tdp_stats *out);

/* ---- refine seam ------------------------------------------------------------
 * Drop-in for the reference's batched refine (MeshDist_batch_gpu_op_shm_flat_stream):
 *   data        9 floats per triangle (3 vertices), element_num triangles   (host)
 *   hausdorff   2 floats per triangle: (proxy-hausdorff, hausdorff), or NULL (host)
 *   offset_size 4 size_t per voxel pair: (off1, n1, off2, n2) in triangles (host)
 *   out         3 floats per voxel pair (host):
 *               distance = min TriDist, min_dist = min max(d-ph1-ph2, 0),
 *               max_dist = min d+h1+h2   (FLT_MAX where a side is empty; with
 *               hausdorff == NULL, min_dist = max_dist = FLT_MAX like the reference)
 * form: TDP_FORM_PLAIN (one CTA per voxel pair) or TDP_FORM_TUNED (persistent,
 * warp-cooperative, culled).  Both return the same minima up to FP32 rounding. */
enum { TDP_FORM_PLAIN = 0, TDP_FORM_TUNED = 1 };
int tdp_refine_batch(tdp_ctx *ctx, const float *data, const float *hausdorff, size_t element_num,
                     const size_t *offset_size, uint32_t pair_num, int form, float *out);

#ifdef __cplusplus
}
#endif
#endif /* TDP_H */
