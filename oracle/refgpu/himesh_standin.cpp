/*
 * himesh_standin.cpp -- test infrastructure, not product code.
 *
 * Definitions behind himesh_standin.h for the reference's GPU-join build:
 * the query context the reference defines in a CGAL source
 * (src/spatial/himesh_query.cpp:13), and HiMesh members that exist only for
 * COMPRESSED / MULTIMESH tiles or the CPU AABB-tree path, none of which a
 * RAW tile reaches.  Each stops the program with a message if called.
 */
#include "himesh_standin.h"

#include <cstdio>
#include <cstdlib>

namespace tdbase {

query_context global_ctx;

namespace {
[[noreturn]] void unsupported(const char* what) {
    std::fprintf(stderr, "reference GPU join build: %s needs CGAL meshes (RAW tiles only)\n", what);
    std::exit(3);
}
}  // namespace

HiMesh::HiMesh(char*, size_t, bool) { unsupported("HiMesh(data)"); }
HiMesh::~HiMesh() {}
void HiMesh::decode(int) { unsupported("HiMesh::decode"); }
size_t HiMesh::fill_voxels(vector<Voxel*>&) { unsupported("HiMesh::fill_voxels"); }
float HiMesh::getHausdorffDistance() { unsupported("HiMesh::getHausdorffDistance"); }
float HiMesh::getProxyHausdorffDistance() { unsupported("HiMesh::getProxyHausdorffDistance"); }
void* HiMesh::get_aabb_tree_triangle() { unsupported("HiMesh::get_aabb_tree_triangle"); }
void* HiMesh::get_segments() { unsupported("HiMesh::get_segments"); }
void HiMesh::clear_aabb_tree() { unsupported("HiMesh::clear_aabb_tree"); }
float HiMesh::distance_tree(HiMesh*) { unsupported("HiMesh::distance_tree"); }
bool HiMesh::intersect_tree(HiMesh*) { unsupported("HiMesh::intersect_tree"); }
aab HiMesh::get_mbb() { unsupported("HiMesh::get_mbb"); }
size_t HiMesh::fill_vertices(float*&) { unsupported("HiMesh::fill_vertices"); }
size_t HiMesh::size_of_triangles() { unsupported("HiMesh::size_of_triangles"); }
size_t HiMesh::get_data_size() { unsupported("HiMesh::get_data_size"); }
const char* HiMesh::get_data() { unsupported("HiMesh::get_data"); }
vector<Voxel*> HiMesh::generate_voxels_skeleton(int) { unsupported("HiMesh::generate_voxels_skeleton"); }
pair<float, float> HiMesh::computeHausdorfDistance(HiMesh*) { unsupported("HiMesh::computeHausdorfDistance"); }
void HiMesh::computeHausdorfDistance() { unsupported("HiMesh::computeHausdorfDistance"); }
pair<float, float> HiMesh::collectGlobalHausdorff() { unsupported("HiMesh::collectGlobalHausdorff"); }
void HiMesh::encode() { unsupported("HiMesh::encode"); }
string HiMesh::to_wkt() { unsupported("HiMesh::to_wkt"); }

}  // namespace tdbase
