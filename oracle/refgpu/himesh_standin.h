/*
 * himesh_standin.h -- test infrastructure, not product code.
 *
 * A CGAL-free declaration of the mesh types that the reference's join, tile
 * and RAW-wrapper sources name, so that those sources (unmodified, compiled
 * where they lie) build the reference's own GPU join as a comparison
 * baseline.  Pre-included with -include, it defines the include guard of the
 * reference's src/include/himesh.h, whose CGAL types cannot be built here, so
 * that header is skipped.  HiMesh_Wrapper keeps the fields and methods of the
 * reference declaration (src/include/himesh.h:688-777) that the join reads;
 * the methods themselves come from the reference's
 * src/spatial/himesh_wrapper.cpp.  Only RAW tiles are supported: HiMesh is an
 * empty type whose members (used only by the COMPRESSED and MULTIMESH modes
 * and by the CPU AABB-tree path) abort when called (himesh_standin.cpp).
 */
#ifndef PROGRESSIVEPOLYGONS_MYMESH_H
#define PROGRESSIVEPOLYGONS_MYMESH_H

#include <assert.h>
#include <pthread.h>
#include <stdint.h>

#include <atomic>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <list>
#include <map>
#include <string>
#include <vector>

#include "aab.h"
#include "geometry.h"
#include "query_context.h"
#include "util.h"

namespace tdbase {
using namespace std;

enum Decoding_Type { COMPRESSED = 0, RAW = 1, MULTIMESH = 2 };

class HiMesh {
public:
    HiMesh(char* data, size_t dsize, bool own_data);
    ~HiMesh();
    void decode(int lod = 100);
    size_t fill_voxels(vector<Voxel*>& voxels);
    float getHausdorffDistance();
    float getProxyHausdorffDistance();
    void* get_aabb_tree_triangle();
    void* get_segments();
    void clear_aabb_tree();
    float distance_tree(HiMesh* target);
    bool intersect_tree(HiMesh* target);
    aab get_mbb();
    size_t fill_vertices(float*& vertices);
    size_t size_of_triangles();
    size_t get_data_size();
    const char* get_data();
    vector<Voxel*> generate_voxels_skeleton(int voxel_size = 100);
    pair<float, float> computeHausdorfDistance(HiMesh* original);
    void computeHausdorfDistance();
    pair<float, float> collectGlobalHausdorff();
    void encode();
    string to_wkt();
};

class HiMesh_Wrapper {
public:
    map<int, float> hausdorffs;
    map<int, float> proxyhausdorffs;
    map<int, HiMesh*> meshes;
    HiMesh* mesh = NULL;
    float transform[3];
    Decoding_Type type;
    size_t id = -1;
    weighted_aab box;
    vector<Voxel*> voxels;
    char* data_buffer = NULL;
    size_t data_size = 0;
    char* meta_buffer = NULL;
    size_t meta_size = 0;
    pthread_mutex_t lock;
    vector<HiMesh_Wrapper*> results;
    int cur_lod = -1;

    HiMesh_Wrapper(map<int, HiMesh*>& meshes);
    HiMesh_Wrapper(HiMesh* mesh);
    HiMesh_Wrapper(char* dt, size_t id, Decoding_Type t = COMPRESSED);
    ~HiMesh_Wrapper();

    HiMesh* get_mesh() {
        if (type == COMPRESSED) return mesh;
        if (type == MULTIMESH) return meshes[cur_lod];
        assert(false);
        return NULL;
    }
    map<int, HiMesh*> get_meshes() { return meshes; }
    void decode_to(int lod);
    void clear_voxels();
    size_t get_voxel_offset(int id, int lod);
    size_t get_voxel_size(int id, int lod);
    float getHausdorffDistance();
    float getProxyHausdorffDistance();
    void report_result(HiMesh_Wrapper* result);
};

}  // namespace tdbase

#endif
