// gen_capi.cpp -- C ABI of the tile generator (include/tdp.h, "synthetic tiles").
#include <cstring>
#include <string>

#include "storage/gen.h"
#include "tdp.h"

extern "C" {

void tdp_gen_default_params(tdp_gen_params* p) {
    if (!p) return;
    tdp::GenParams d;
    p->n_vessels = d.n_vessels;
    p->nuclei_per_vessel = d.nuclei_per_vessel;
    p->seed = d.seed;
    p->voxel_size = d.voxel_size;
    p->nucleus_subdiv = d.nucleus_subdiv;
    p->tube_sides = d.tube_sides;
    p->tube_rings = d.tube_rings;
    p->threads = d.threads;
    p->grid = d.grid;
    p->shell_min = d.shell_min;
    p->shell_max = d.shell_max;
    p->nuclei_begin = 0;
    p->nuclei_end = 0;
}

namespace {

tdp::GenParams to_gen(const tdp_gen_params* p) {
    tdp::GenParams g;
    g.n_vessels = p->n_vessels;
    g.nuclei_per_vessel = p->nuclei_per_vessel;
    g.seed = p->seed;
    g.voxel_size = p->voxel_size;
    g.nucleus_subdiv = p->nucleus_subdiv;
    g.tube_sides = p->tube_sides;
    g.tube_rings = p->tube_rings;
    g.threads = p->threads;
    g.grid = p->grid;
    g.shell_min = p->shell_min;
    g.shell_max = p->shell_max;
    g.nuclei_begin = p->nuclei_begin;
    g.nuclei_end = p->nuclei_end;
    return g;
}

int report(int rc, const std::string& msg, char* err, size_t err_cap) {
    if (rc != TDP_OK && err && err_cap) {
        std::strncpy(err, msg.c_str(), err_cap - 1);
        err[err_cap - 1] = 0;
    }
    return rc;
}

}  // namespace

int tdp_gen_tiles(const tdp_gen_params* p, uint8_t* nuclei, size_t nuclei_cap, size_t* nuclei_len,
                  uint8_t* vessels, size_t vessels_cap, size_t* vessels_len, char* err, size_t err_cap) {
    if (!p) return TDP_ERR_ARG;
    std::string msg;
    const int rc = tdp::gen_tiles(to_gen(p), nuclei, nuclei_cap, nuclei_len, vessels, vessels_cap, vessels_len, msg);
    return report(rc, msg, err, err_cap);
}

int tdp_gen_meshes(const tdp_gen_params* p, int which, float* vertices, size_t vert_cap, int64_t* vert_off,
                   uint32_t* faces, size_t face_cap, int64_t* face_off, size_t* n_vert, size_t* n_face,
                   long* n_obj, char* err, size_t err_cap) {
    if (!p) return TDP_ERR_ARG;
    std::string msg;
    const int rc = tdp::gen_meshes(to_gen(p), which, vertices, vert_cap, vert_off, faces, face_cap, face_off, n_vert,
                                   n_face, n_obj, msg);
    return report(rc, msg, err, err_cap);
}

}  // extern "C"
