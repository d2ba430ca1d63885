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
 * hold (0 = no cap beyond what the device has).  flags: 0, or TDP_CTX_POISON:
 * the triangle records of attached tiles start as NaN instead of whatever the
 * allocation held, so that a read of a record no fetch filled shows in the
 * results (for tests; it costs a memset of the records per attach). */
#define TDP_CTX_POISON 1u
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
    double candidates_ms;            /* host wall time of object candidates     */
    double lod_ms;                   /* device time of the LOD loop             */
    long host_syncs;                 /* host<->device synchronisations          */
    double exact_ms;                 /* exact-distance stage (device time)      */
    long exact_items;                /* LOD-100 voxel pairs it refined in FP32  */
    long exact_f64_items;            /* of those, evaluated in FP64             */
    double fp32_max_rel_err;         /* exact stage: max |FP32 minimum - FP64
                                        distance| / max(distance, 1)           */
    double fetch_bytes;              /* RAW bytes fetched from attached tiles
                                        (tdp_tile_attach) during the call     */
    long lod_graph;                  /* tuned LOD loop: 0 launched directly,
                                        1 replayed the context's CUDA graph,
                                        2 captured (or updated) it in this call */
    double refine_ms_lod[5];         /* tuned refine time per LOD 20..100      */
    double exact_phase_ms[4];        /* exact stage, device time of: upper
                                        bounds (with their FP32 refine),
                                        candidate voxel pairs, the FP32 pass,
                                        the FP64 pass                          */
    unsigned long long exact_full_evals; /* exact stage: triangle pairs fully
                                        evaluated by its FP32 pass             */
    long candidates_on_device;       /* 1: object candidates were computed on
                                        the GPU (tuned form), 0: on the host   */
    long candidate_redone;           /* kNN queries whose ring search outgrew a
                                        warp's shared-memory buffer and were
                                        redone on the GPU with a global one    */
    long exact_dropped_items;        /* exact stage: FP32-pass voxel pairs
                                        dropped by the refine's item-level
                                        bound test (no triangle staged)        */
    long exact_below_items;          /* exact stage: FP32-pass voxel pairs with
                                        a triangle pair below their preset     */
} tdp_stats;
int tdp_last_stats(const tdp_ctx *ctx, tdp_stats *out);
/* measured FP32 FMA throughput of the context's device in TFLOP/s (CUDA cores,
 * no tensor cores): the roofline ceiling of the refine kernels. */
int tdp_fp32_peak(tdp_ctx *ctx, double *tflops);
/* ---- tuned refine configurations --------------------------------------
 * The tuned refine kernel exists in a few configurations: A-side triangles
 * staged per warp and resident CTAs per SM (configurations 0-2 stage each
 * triangle's full pre-processed record in shared memory; 3-7 stage only its
 * bounds and pre-process the triangles of each evaluated pair in registers;
 * 8-9 do the same with one lane per evaluated pair; 10-11 are 6 and 9 queuing
 * only the 8 most promising first pairs before the cull; 12-13 stage each
 * chunk's triangle records in shared memory by a 1-D bulk copy (TMA); 14-15
 * spread each needed cluster's member tests over the warp; 16-17 are 14-15
 * with a cylinder bound -- gap along the item's axis, centre distance across
 * it less both radii -- in every cull test).  All return identical results;
 * they differ only in speed, which depends on the voxel sizes of the join.
 * A context starts with configuration 0.  The reference has one fixed launch
 * shape (one CTA of 512 threads per voxel pair,
 * MeshDist_batch_gpu_op_shm_flat_stream, src/geometry/computing_gpu.cu:6540-6658)
 * and no counterpart to these calls. */
int tdp_refine_config_count(void);
int tdp_refine_config_info(int cfg, int *chunk_a, int *ctas_per_sm);
int tdp_set_refine_config(tdp_ctx *ctx, int cfg);
int tdp_get_refine_config(const tdp_ctx *ctx, int *cfg);
/* The configuration the tuned form uses at one LOD (20, 40, 60, 80, 100):
 * tdp_autotune keeps, besides the fastest configuration over the whole join
 * (its *best), the fastest one at each LOD, and the LOD loop launches each
 * LOD's own; tdp_set_refine_config sets one configuration for every LOD. */
int tdp_get_refine_config_lod(const tdp_ctx *ctx, int lod, int *cfg);

/* ---- CUDA graph of the LOD loop --------------------------------------
 * The tuned form's LOD loop (per LOD: item build, refine, bound update,
 * decision; then the FP64 recheck) is a fixed sequence of about 30 launches
 * whose counts stay in device memory.  A context can capture it as a CUDA
 * graph and replay it while the loop's launch arguments (tiles, buffers,
 * voxel-pair count, LOD list, query, refine configuration) stay the same:
 *   TDP_LOD_GRAPH_OFF     launch directly, always;
 *   TDP_LOD_GRAPH_AUTO    (default) capture arguments on their second use, so
 *                         one-off joins (served batches) launch directly and
 *                         repeated joins replay the graph;
 *   TDP_LOD_GRAPH_ALWAYS  capture whenever the arguments change.
 * Results are identical in every mode.  No reference counterpart: the
 * reference launches and synchronises per chunk and per LOD
 * (src/join/KNNJoin.cpp:1596-1714). */
enum { TDP_LOD_GRAPH_OFF = 0, TDP_LOD_GRAPH_AUTO = 1, TDP_LOD_GRAPH_ALWAYS = 2 };
int tdp_set_lod_graph(tdp_ctx *ctx, int mode);

/* The context's CUDA stream (a cudaStream_t), on which every tdp call that
 * takes this context launches its work: callers order their own work, or
 * record timing events, against it.  NULL for a NULL context. */
void *tdp_ctx_stream(const tdp_ctx *ctx);

/* ---- tiles ------------------------------------------------------------------
 * Upload a RAW .dt tile (the bytes of the file, host memory, pinned or not)
 * into HBM: voxel records and every LOD's triangles become resident.
 * max_objects <= 0 loads all objects (reference --max_objects1/2).
 * Errors: TDP_ERR_FORMAT for malformed bytes, TDP_ERR_NOMEM over budget. */
typedef struct {
    long n_objects;
    long n_voxels;
    long n_tris[5];        /* per LOD 20,40,60,80,100 */
    size_t device_bytes;
    size_t h2d_bytes;      /* bytes the upload / attach itself copied host -> device */
    int attached;          /* 1 for a tile made by tdp_tile_attach */
    double parse_ms;       /* host time of the upload / attach: parsing the bytes
                              (the parser writes the voxel records into the
                              page-locked staging buffer),                        */
    double alloc_ms;       /* allocating the device arrays,                       */
    double load_ms;        /* and in total                                        */
    double meta_ms;        /* of which the prefix sums, the rest of the staging
                              and the copies of the metadata to the device (for
                              an attach: queuing them, not their completion)      */
} tdp_tile_info;
int tdp_tile_upload(tdp_ctx *ctx, const void *raw_dt, size_t len, long max_objects, tdp_tile **out);
/* Attach a RAW tile that stays in page-locked host memory (cudaHostRegister or
 * cudaHostAlloc covering all len bytes; it must outlive the tile): only the
 * voxel and object metadata are copied now (the call may return with those
 * copies still queued on the context's stream, tdp_ctx_stream, which every
 * later call on the context is ordered after); each join copies, LOD by LOD, the
 * triangles of the voxels its refine touches, straight from the host bytes,
 * and keeps them for later joins on the tile.  This is the reference's
 * per-LOD staging of the voxels a chunk needs (build_chunks_by_pair /
 * packing_data_stream, src/join/KNNJoin.cpp:1473-1521,
 * src/join/SpatialJoin.cpp:169-248) done by the GPU.  Results equal those of
 * an uploaded tile.  The tile must be in the writer's layout (each object's
 * data block LOD by LOD, voxel by voxel: src/storage/tile_IO.cpp:79-172),
 * else TDP_ERR_FORMAT; unlocked memory is TDP_ERR_ARG. */
int tdp_tile_attach(tdp_ctx *ctx, const void *raw_dt, size_t len, long max_objects, tdp_tile **out);
/* Validate RAW tile bytes on the host (no device needed): the same
 * bounds-checked parser the uploads use.  TDP_ERR_FORMAT with the first
 * problem in file order described in err (NUL-terminated, err_len bytes). */
int tdp_raw_check(const void *raw, size_t len, long *n_objects, long *n_voxels, char *err, size_t err_len);
/* page-locked host memory (cudaHostAlloc) to read tiles into for attaching */
int tdp_host_alloc(size_t bytes, void **out);
int tdp_host_free(void *p);
/* The parser's large host arrays (1 MiB and up) are recycled through a
 * process-wide cache of freed blocks, at most 4 GiB: repeated uploads and
 * attaches then pay no page faults on fresh memory.  No reference
 * counterpart.  tdp_host_cache_bytes: freed bytes the cache holds now;
 * tdp_host_cache_trim: hand them all back to the system. */
size_t tdp_host_cache_bytes(void);
void tdp_host_cache_trim(void);
int tdp_tile_free(tdp_ctx *ctx, tdp_tile *tile);
int tdp_tile_get_info(const tdp_tile *tile, tdp_tile_info *out);

/* ---- bound preparation (GPU) ------------------------------------------------
 * Replaces the reference's CGAL preparation of the per-triangle bounds the join
 * reads (sampled in src/spatial/himesh_hausdorff.cpp:197-270, stored as
 * (proxy, hausdorff) per triangle at src/spatial/himesh_retrieve.cpp:131-151,
 * written by tdbase convert through src/storage/tile_IO.cpp:79-172) with a
 * conservative rule computed on the GPU in FP64 from each object's own LOD-100
 * surface S:
 *   proxy ph(t): every LOD-100 facet goes to the LOD triangle nearest its
 *     barycentre; ph(t) = the largest distance of an assigned facet's vertex
 *     to t, so every point of S lies within ph of its triangle;
 *   hausdorff h(t): t cut into up to 64 pieces about one LOD-100 edge long;
 *     h(t) = the largest over pieces of the smallest over facets of the
 *     largest corner distance, so every point of t lies within h of S;
 * rounded up to float; the object-level values are the per-LOD maxima (LOD
 * 100: 0).  The triangles, voxels and LODs themselves are the input's.
 * tdp_tile_compute_bounds rewrites the bounds of a resident tile in place (a
 * join may use it at once); tdp_raw_compute_bounds maps RAW bytes to RAW
 * bytes (out: len bytes, may equal raw) through a temporary resident tile. */
typedef struct {
    double ms;           /* device time of the bound kernels (CUDA events) */
    long objects;        /* objects of the tile */
    long triangles;      /* LOD 20-80 triangles bounded */
    long facet_queries;  /* (LOD-100 facet, LOD) nearest-triangle searches */
    long pieces;         /* triangle pieces searched for their nearest facet */
    double dist_evals;   /* FP64 point-to-triangle distances evaluated */
} tdp_bounds_info;
int tdp_tile_compute_bounds(tdp_ctx *ctx, tdp_tile *tile, tdp_bounds_info *info);
int tdp_raw_compute_bounds(tdp_ctx *ctx, const void *raw, size_t len, void *out, tdp_bounds_info *info);

/* ---- LOD preparation (GPU) --------------------------------------------------
 * Replaces the reference's CGAL preparation of a tile from LOD-100 meshes (the
 * OFF polyhedra of its data/ prototypes): progressive decimation into LODs
 * (src/spatial/himesh_comp.cpp:28-190), skeleton voxels
 * (src/spatial/himesh_skeleton.cpp:17-168), LOD triangles to voxels
 * (src/spatial/himesh_retrieve.cpp:183-200), the Hausdorff bounds and the RAW
 * writer of tdbase convert (src/storage/tile_IO.cpp:79-172).  Every step runs
 * on the GPU (csrc/prep_kernels.cu states the rule): LODs 80/60/40/20 by
 * shortest-edge half-edge collapse, voxels of about voxel_size LOD-100 facets
 * by farthest-point seeds and two Lloyd steps, triangles to the voxel with the
 * nearest core, then the bounds of tdp_raw_compute_bounds.
 * Object o: vertices[3 vert_off[o] .. 3 vert_off[o+1]) (x, y, z floats) and
 * facets faces[3 face_off[o] .. 3 face_off[o+1]) (vertex indices local to the
 * object); vert_off and face_off hold n_objects + 1 non-decreasing entries.
 * out receives the RAW tile (*len bytes); cap >= the size tdp_raw_prep_bound
 * gives always suffices; out = NULL only computes *len.  TDP_ERR_ARG names
 * the first object without vertices or facets, with an index out of range, a
 * facet repeating a vertex or a non-finite coordinate. */
typedef struct {
    double total_ms;      /* host wall time of the call */
    double decimate_ms;   /* device time of the decimation kernels */
    double voxel_ms;      /* device time of the voxel kernel */
    double write_ms;      /* device time of the RAW writer */
    double bounds_ms;     /* host wall time of the bound preparation */
    long n_objects;
    long n_triangles[5];  /* per LOD 20..100 */
    long n_voxels;
    long batches;         /* object batches the call was split into */
} tdp_prep_info;
int tdp_raw_prep_bound(const int64_t *face_off, long n_objects, int voxel_size, size_t *max_len);
int tdp_raw_from_meshes(tdp_ctx *ctx, const float *vertices, const int64_t *vert_off, const uint32_t *faces,
                        const int64_t *face_off, long n_objects, int voxel_size, void *out, size_t cap,
                        size_t *len, tdp_prep_info *info);

/* ---- object candidates (host only) ------------------------------------------
 * The object-level filter: replaces OctreeNode::query_knn_fast / query_within
 * over Tile::build_octree (reference src/index/octree.cpp:215-330,
 * src/storage/tile.cpp:76-85).  Boxes are 6 floats (low xyz, high xyz),
 * transforms 3 floats.  kNN (is_knn == 1): the knn objects with the smallest
 * transform distance plus every object whose box gap is below the knn-th of
 * those distances, ordered by (transform distance, id).  within (is_knn == 0):
 * every object with box gap <= within, ordered by id.  intersect (is_knn == 2,
 * OctreeNode::query_intersect, src/index/octree.cpp:332-349): every object
 * whose box overlaps strictly, ordered by id.  self_join excludes the query
 * object.
 * off: [n1+1] CSR offsets.  Returns the number of candidates, or -(needed) when
 * cap is too small (off is then valid, ids is not), LONG_MIN on bad arguments. */
long tdp_candidates(const float *box1, const float *xf1, long n1, const float *box2, const float *xf2, long n2,
                    int self_join, int is_knn, int knn, float within, int64_t *off, int32_t *ids, long cap);
/* The same candidates computed on the GPU for two resident tiles (tile2 NULL or
 * == tile1: self-join); this is what the tuned join uses.  A kNN query whose
 * ring search outgrows a warp's shared-memory buffer (large K, dense cells) is
 * redone on the GPU with a global buffer; the number of such queries is then
 * tdp_last_stats().candidate_redone.  Same return convention as
 * tdp_candidates; LONG_MIN on error (see tdp_last_error). */
long tdp_tile_candidates(tdp_ctx *ctx, const tdp_tile *tile1, const tdp_tile *tile2, int is_knn, int knn,
                         float within, int64_t *off, int32_t *ids, long cap);

/* ---- splitting a join over GPUs ------------------------------------------------
 * No reference counterpart (the reference pins itself to one GPU,
 * src/geometry/cuda_common.cu:20).  A join's query objects are independent
 * given tile 2: each query object's candidate list, filter and LOD refine read
 * only that object and tile 2 (per-object candidate lists,
 * src/join/KNNJoin.cpp:552-600).  So N processes, one per GPU, can each join a
 * contiguous range of tile-1 objects (tdp_join_params.query_begin/query_end)
 * against the whole tile 2 and concatenate their results, with no exchange
 * during the join.  tdp_partition_queries splits [0, n1) into n_shards
 * contiguous ranges of about equal estimated work: per query object, the sum
 * over its object candidates (as tdp_candidates returns them) of
 * n_voxels(query) x n_voxels(candidate) -- the voxel pairs the filter
 * evaluates -- plus one.  bounds receives n_shards + 1 entries (bounds[0] = 0,
 * bounds[n_shards] = n1; shard s is [bounds[s], bounds[s+1]), possibly
 * empty); work (optional) each shard's estimate.  is_knn: 0 within, 1 kNN,
 * 2 intersect.  Host only, deterministic: every process computes the same
 * split from the same inputs. */
int tdp_partition_queries(const float *box1, const float *xf1, const uint32_t *nvox1, long n1,
                          const float *box2, const float *xf2, const uint32_t *nvox2, long n2,
                          int self_join, int is_knn, int knn, float within, int n_shards,
                          long *bounds, double *work);
/* The same from RAW tiles in host memory, parsed on the host (raw2 NULL: a
 * self-join of raw1).  err (optional) receives a message. */
int tdp_raw_partition(const void *raw1, size_t len1, const void *raw2, size_t len2, int is_knn, int knn,
                      float within, int n_shards, long *bounds, double *work, char *err, size_t err_cap);

/* ---- join ---------------------------------------------------------------------
 * `tdbase join` (reference src/tools/tdbase.cpp:482-549) on device-resident tiles:
 * object candidates (grid restatement of the octree queries), voxel-pair filter,
 * then the LOD loop of refine + bound update + decision.  tile2 == NULL or
 * tile2 == tile1 is a self-join (query object excluded from its own candidates;
 * within results then hold both (a,b) and (b,a), as in the reference).
 * Results are (query id, result id) pairs sorted by query then result id. */
/* TDP_QUERY_INTERSECT (-q intersect, SpatialJoin::intersect,
 * src/join/IntersectionJoin.cpp:12-140 with TriInt_cuda,
 * src/geometry/computing_gpu.cu:1441-1511): candidates are objects whose boxes
 * overlap strictly (aab::intersect, src/spatial/himesh_box.cpp:95-99), voxel
 * pairs likewise; a pair is reported when a voxel pair's max_dist = min(d + h1
 * + h2) is 0 and dropped when every voxel pair's min_dist is above 0 -- the
 * decisions of a within join at distance 0, with LOD 100 deciding. */
enum { TDP_QUERY_NN = 1, TDP_QUERY_WITHIN = 2, TDP_QUERY_INTERSECT = 3 };
typedef struct {
    int query;             /* TDP_QUERY_NN (-q nn), TDP_QUERY_WITHIN (-q within) or
                              TDP_QUERY_INTERSECT (-q intersect; within_dist unused) */
    int knn;               /* --knn K                      (default 1)             */
    float within_dist;     /* --within_dist tau            (default 1000)          */
    int lods[8];           /* -l/--lods, ascending; n_lods = 0 -> 20,40,60,80,100  */
    int n_lods;
    int hausdorff_level;   /* --hausdorff_level 0|1|2      (default 2)             */
    int form;              /* TDP_FORM_PLAIN (reference decision rules in FP32) or
                              TDP_FORM_TUNED (persistent refine, FP32 with error
                              bands and an FP64 recheck of undecided pairs)        */
    int exact_distances;   /* 1: give every result its LOD-100 distance in FP64
                              (tdp_result_copy_f64); the reference reports ids
                              only, so this stage has no counterpart (default 0) */
    const int *obj_knn;    /* NULL, or one entry per tile-1 object: K (> 0, that
                              object is a kNN query) or 0 (a within query at
                              distance obj_within[i]).  Lets one join carry a
                              batch of different requests; query/knn/within_dist
                              are then ignored.  No reference counterpart. */
    const float *obj_within;
    long query_begin;      /* join only tile-1 objects [query_begin, query_end)     */
    long query_end;        /* (query_end < 0: to the last one; default 0, -1); result
                              ids stay tile-1 ids and a self-join still excludes
                              each object itself.  One shard of a join split over
                              GPUs (tdp_partition_queries).  No reference
                              counterpart: the reference runs on one GPU
                              (src/geometry/cuda_common.cu:20). */
} tdp_join_params;
void tdp_join_default_params(tdp_join_params *p);
int tdp_join(tdp_ctx *ctx, const tdp_tile *tile1, const tdp_tile *tile2, const tdp_join_params *p,
             tdp_result **out);
int tdp_result_count(const tdp_result *r, long *n);
/* any output pointer may be NULL; dist = the pair's upper distance bound when
 * it was decided (the exact FP32 distance for pairs decided at the last LOD) */
int tdp_result_copy(const tdp_result *r, int *query_ids, int *result_ids, float *dist);
/* the exact LOD-100 distances (double, minimum over the stored float
 * coordinates up to FP64 rounding), in the same row order; TDP_ERR_STATE when
 * the join ran without exact_distances */
int tdp_result_copy_f64(const tdp_result *r, double *dist);
int tdp_result_free(tdp_result *r);

/* Autotuner: runs the tuned join of `params` once per configuration untimed
 * and once timed, keeps the configuration with the least refine time for the
 * context and returns it in *best (may be NULL).  ms_per_config, if not NULL,
 * receives tdp_refine_config_count() refine times in milliseconds. */
int tdp_autotune(tdp_ctx *ctx, const tdp_tile *tile1, const tdp_tile *tile2, const tdp_join_params *params,
                 double *ms_per_config, int *best);

/* ---- joins larger than the device ------------------------------------------
 * Joins host RAW tiles that need not fit on the device (config 4: a device
 * budget below the tiles' size).  The candidates are computed on the host for
 * the whole tiles; tile 1 is joined in chunks of chunk_objects query objects,
 * each against a sub-tile of tile 2 holding exactly that chunk's candidates.
 * The result equals tdp_join on the whole tiles (ids and distances).  Chunks
 * hold at most chunk_objects query objects and, when the context has a
 * budget, are cut so that the chunk, its sub-tile and the join's scratch fit
 * it (estimated from their RAW bytes; a chunk that still runs out of device
 * memory is split in two and retried).  No per-object queries;
 * tile 2 must be a different tile (no self-join).  No reference counterpart
 * (the reference keeps both tiles decoded in host memory and sizes its device
 * scratch for the whole tile, src/geometry/computing_gpu.cu:4538-4626). */
typedef struct {
    long chunks;
    long splits;               /* chunks split in two after running out of memory        */
    double h2d_bytes;          /* bytes copied host -> device: chunk and sub-tile
                                  metadata plus the triangles the joins fetched (chunks
                                  are assembled in page-locked buffers and attached;
                                  whole uploads when page-locking is unavailable)     */
    double tri_pairs;          /* refined triangle pairs, all chunks                      */
    double join_ms;            /* device time of the chunk joins                          */
    double device_peak_bytes;  /* the context's device-memory high-water mark             */
} tdp_chunked_info;
int tdp_join_chunked(tdp_ctx *ctx, const void *raw1, size_t len1, const void *raw2, size_t len2,
                     const tdp_join_params *p, long chunk_objects, tdp_chunked_info *info, tdp_result **out);

/* ---- serving ------------------------------------------------------------------
 * A request loop over one resident tile 2 (for example the vessel tile): each
 * request is a RAW .dt tile of query objects with its own query (kNN with its
 * own K, or within with its own distance).  Requests are admitted into one of
 * two device arenas as long as they fit its capacity (admission by memory);
 * while the GPU joins one arena, newly arriving requests are copied into the
 * other on a separate stream, and when the running batch ends the next one
 * starts with every request admitted meanwhile (continuous batching).  A batch
 * is one tdp_join whose query objects carry their requests' own queries
 * (obj_knn / obj_within), so each request's result equals the result of
 * tdp_join on that request alone.
 * The reference runs one join per invocation of `tdbase join`
 * (src/tools/tdbase.cpp:482-549) and has no request loop: no counterpart.
 *
 * The server takes over the context: no other call may use `ctx` until
 * tdp_server_destroy.  The bytes passed to tdp_server_submit must stay valid
 * until that request completes (tdp_server_wait returned TDP_OK or an error).
 * Requests in page-locked memory (cudaHostRegister / cudaHostAlloc, e.g.
 * tdp_host_alloc) stage only their metadata: the batch join fetches, per
 * LOD, the triangles of the voxels it refines straight from their bytes;
 * other requests are copied whole. */
typedef struct tdp_server tdp_server;
typedef struct {
    long arena_objects;        /* query objects one arena holds        (default 65536)    */
    long arena_voxels;         /* voxels one arena holds               (default 2^20)     */
    long arena_tris;           /* triangles per LOD one arena holds    (default 2^25)     */
    size_t max_request_bytes;  /* largest RAW request accepted         (default 1 GiB)    */
    int lods[8];               /* LOD list as in tdp_join_params (n_lods = 0: all)        */
    int n_lods;
    int hausdorff_level;       /* default 2 */
    int form;                  /* default TDP_FORM_TUNED */
    double big_request_ms;     /* a batch that mixes requests estimated above this join
                                  time with smaller ones runs as two joins, the small
                                  requests first, each request done with its own pass
                                  (default 4; <= 0: one join per batch)                  */
} tdp_server_params;
typedef struct {
    double queue_ms;           /* submit -> its batch started                              */
    double latency_ms;         /* submit -> result ready                                   */
    long batch;                /* index of the batch that served it                        */
    int batch_requests;        /* requests in that batch                                    */
    int status;                /* TDP_OK, or why the request failed                        */
} tdp_request_info;
typedef struct {
    long batches;
    long requests;             /* completed (including failed)                             */
    long failed;
    double busy_ms;            /* wall time the executor spent in joins                    */
    double upload_ms;          /* per request, staging copy start to arena append done,
                                  summed (the copies of two requests overlap)              */
    double upload_bytes;       /* bytes staged: every request's metadata, and the RAW bytes
                                  of requests not in page-locked memory                    */
    double fetch_bytes;        /* RAW bytes the batch joins fetched from page-locked
                                  requests (only the voxels they refined)                  */
    long split_batches;        /* batches run as a small pass and a big pass               */
} tdp_server_stats;
void tdp_server_default_params(tdp_server_params *p);
/* allocates both arenas in the context (counted against its budget) */
int tdp_server_create(tdp_ctx *ctx, const tdp_tile *tile2, const tdp_server_params *p, tdp_server **out);
/* query: TDP_QUERY_NN (knn >= 1) or TDP_QUERY_WITHIN (within >= 0).  The bytes
 * are parsed here: TDP_ERR_FORMAT for malformed bytes, TDP_ERR_ARG for a request
 * larger than an arena or than max_request_bytes. */
int tdp_server_submit(tdp_server *srv, const void *raw_dt, size_t len, int query, int knn, float within,
                      uint64_t *request_id);
/* Waits up to timeout_ms (< 0: no limit) for the request; TDP_ERR_TIMEOUT if it
 * is not done yet (call again).  On completion returns its status and, when
 * TDP_OK, the result with the request's own object ids (tdp_result_* calls;
 * free it with tdp_result_free).  info may be NULL.  A request id can be
 * waited for successfully once. */
int tdp_server_wait(tdp_server *srv, uint64_t request_id, int timeout_ms, tdp_result **result,
                    tdp_request_info *info);
int tdp_server_get_stats(const tdp_server *srv, tdp_server_stats *out);
/* Stops admitting, runs the batches already admitted, fails the requests not
 * yet admitted (TDP_ERR_STATE), frees the arenas and hands the context back. */
int tdp_server_destroy(tdp_server *srv);

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

/* ---- refine without any device allocation -------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a plugin inside an application that owns the GPU's memory pool, a
 * process held to a fixed device budget, a latency-critical loop that must not
 * call cudaMalloc): the same refine as tdp_refine_batch with TDP_FORM_TUNED,
 * but every pointer is DEVICE memory and the call needs no context and
 * allocates nothing.  It runs the tuned kernel's configuration 0 (no
 * autotuner pick applies without a context).  Its working memory is one fixed
 * __device__ array of 14,680,320 bytes (14.0 MiB) inside this library (held by
 * every GPU that loads it until exit), which caps a call at 262144 triangles
 * and 65536 voxel pairs; larger calls return TDP_ERR_ARG with a message in
 * err.  The first call on a device looks up that array's address, and the
 * first launch in a process raises the kernel's dynamic shared-memory limit
 * (make that first call before any stream capture begins).  All calls on a
 * device share the array: calls that may overlap on the GPU race, so serialise
 * them.  Work is enqueued on `stream` (a cudaStream_t, NULL = default stream);
 * out is valid once the stream reaches it.  Rows of offset_size that point
 * outside the batch are not read and yield NaN. */
int tdp_refine_batch_noalloc(const float *data, const float *hausdorff, size_t element_num,
                             const size_t *offset_size, uint32_t pair_num, float *out, void *stream,
                             char *err, size_t err_cap);

/* ---- synthetic tiles (host only, no context) --------------------------------
 * Seeded generator of nuclei/vessel tiles in the reference's RAW .dt format.
 * Replaces the CGAL simulator + `tdbase convert` (reference
 * src/tools/simulator.cpp:332-458, src/storage/tile_IO.cpp:79-172), which cannot
 * be built without CGAL.  Call once with null buffers to learn the sizes, then
 * with buffers of at least those sizes.  err (optional) receives a message. */
typedef struct {
    int n_vessels;          /* vessels, one per cell of a `grid`-unit grid      */
    int nuclei_per_vessel;  /* nuclei in a shell around each vessel             */
    uint64_t seed;
    int voxel_size;         /* target triangles per voxel (100)                 */
    int nucleus_subdiv;     /* icosphere subdivision (3 -> 1280 triangles)      */
    int tube_sides;         /* vessel tube resolution (20 x 72 -> ~20k tris)    */
    int tube_rings;
    int threads;            /* 0 = all hardware threads                         */
    float grid;             /* 1000                                             */
    float shell_min, shell_max; /* 30, 300                                      */
    long nuclei_begin;      /* emit only nuclei [begin, end) of the full tile   */
    long nuclei_end;        /* (end <= 0: all); placement is unchanged          */
} tdp_gen_params;
void tdp_gen_default_params(tdp_gen_params *p);
int tdp_gen_tiles(const tdp_gen_params *p, uint8_t *nuclei, size_t nuclei_cap, size_t *nuclei_len,
                  uint8_t *vessels, size_t vessels_cap, size_t *vessels_len, char *err, size_t err_cap);
/* The LOD-100 meshes of the same objects, as tdp_raw_from_meshes takes them:
 * which = 0 the nuclei [nuclei_begin, nuclei_end), 1 the vessels; float
 * vertices as the tiles store them, the prototype's facets per object.  Null
 * vertices and faces: only n_vert, n_face and n_obj are set. */
int tdp_gen_meshes(const tdp_gen_params *p, int which, float *vertices, size_t vert_cap, int64_t *vert_off,
                   uint32_t *faces, size_t face_cap, int64_t *face_off, size_t *n_vert, size_t *n_face,
                   long *n_obj, char *err, size_t err_cap);

#ifdef __cplusplus
}
#endif
#endif /* TDP_H */
