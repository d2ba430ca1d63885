/*
 * oracle/oracle.h -- TEST INFRASTRUCTURE ONLY (the FP64 checker for the CUDA path).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this.
 */
#ifndef TDP_ORACLE_H
#define TDP_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* triangle-triangle distance, FP64, closest-feature method (see tridist.c) */
double tdo_tri_dist(const double *S9, const double *T9);
/* independent FP64 formulation used to cross-check tdo_tri_dist */
double tdo_tri_dist_features(const double *S9, const double *T9);
void tdo_tri_dist_batch(const double *S, const double *T, size_t n, double *out_pqp, double *out_feat);
/* MeshDist restated in FP64: out = {distance, min low bound, min high bound} */
void tdo_voxel_pair(const float *tri1, const float *hd1, size_t n1,
                    const float *tri2, const float *hd2, size_t n2, double out[3]);

/* per-triangle Hausdorff bounds of a RAW tile (bounds_oracle.cpp): out = a
 * copy of the tile with the bounds replaced; prune 0 = brute force */
int tdo_tile_bounds(const uint8_t *raw, size_t len, uint8_t *out, int prune, int threads, double *evals);
/* largest violation of a tile's bounds over sampled points, see bounds_oracle.cpp */
int tdo_bounds_violation(const uint8_t *raw, size_t len, int samples, uint64_t seed, double out[2]);

/* LOD preparation of meshes into a RAW tile with zero bounds (lodprep_oracle.cpp);
 * 0, -1 for bad arguments or a short buffer, -1 - o for bad object o */
long tdo_raw_from_meshes(const float *vertices, const int64_t *vert_off, const uint32_t *faces,
                         const int64_t *face_off, long n_objects, int voxel_size, uint8_t *out, size_t cap,
                         size_t *len, int threads);

#ifdef __cplusplus
}
#endif
#endif
