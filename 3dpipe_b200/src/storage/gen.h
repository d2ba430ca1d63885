// gen.h -- seeded generator of nuclei / vessel tiles in the reference's RAW format.
//
// The reference generates tiles with CGAL (src/tools/simulator.cpp:332-458) and
// converts them to RAW with `tdbase convert` (src/storage/tile_IO.cpp:79-172);
// CGAL is not available, so this generator restates the definitions the join
// relies on and writes the same RAW layout:
//   * nuclei: icosphere (subdivision 3, 1280 triangles) scaled to an ellipsoid
//     with semi-axes U(8,12), 10 % low-frequency radial noise, random rotation;
//   * vessels: closed tubes of radius U(5,15) swept along a 3-level branching
//     polyline (7 segments, ~20k triangles), one per cell of a 1000-unit grid;
//   * nuclei uniform in a 30-300 unit shell around their vessel, never
//     intersecting each other or a vessel;
//   * LODs 20/40/60/80/100 % by half-edge collapse (LOD vertices are original
//     vertices);
//   * voxels of ~100 triangles by 2-iteration k-means over vertices, facets by
//     barycentre (reference src/spatial/himesh_skeleton.cpp:17-168), lower-LOD
//     triangles to the nearest core by first vertex (himesh_retrieve.cpp:183-200);
//   * per-triangle (proxy-hausdorff, hausdorff) bounds that are conservative by
//     construction (see gen.cpp), object-level maxima, LOD 100 = 0.
// Topology (decimation, voxels, bound assignments) is computed once per
// prototype; each instance only maps vertices and evaluates its bounds, so a
// 200k-nucleus tile is generated in seconds on a few cores.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

namespace tdp {

struct GenParams {
    int n_vessels = 10;
    int nuclei_per_vessel = 20;
    uint64_t seed = 20260001;
    int voxel_size = 100;
    int nucleus_subdiv = 3;
    int tube_sides = 20;
    int tube_rings = 72;
    int threads = 0;           // 0 = hardware concurrency
    float grid = 1000.f;
    float shell_min = 30.f, shell_max = 300.f;
    long nuclei_begin = 0, nuclei_end = 0;  // emit nuclei [begin, end) only (end <= 0: all)
};

// Two-phase: call with null buffers to get the byte sizes, then with buffers of
// at least that size.  Returns 0 or a TDP_ERR_* code (message in err).
int gen_tiles(const GenParams& p, uint8_t* nuclei, size_t nuclei_cap, size_t* nuclei_len, uint8_t* vessels,
              size_t vessels_cap, size_t* vessels_len, std::string& err);

// The LOD-100 meshes of the same objects (which: 0 nuclei [nuclei_begin,
// nuclei_end), 1 vessels): float vertices exactly as the tile stores them and
// the prototype's facets, per object.  Null V and F: sizes only.
int gen_meshes(const GenParams& p, int which, float* V, size_t vcap, int64_t* voff, uint32_t* F, size_t fcap,
               int64_t* foff, size_t* n_vert, size_t* n_face, long* n_obj, std::string& err);

}  // namespace tdp
