/*
 * refgpu_main.cpp -- test infrastructure, not product code.
 *
 * Runs the reference's own join on two RAW tiles through its own classes:
 * the reference's option parser, Tile, geometry_computer (with its GPU
 * refine under -g) and SpatialJoin, in the order the reference's `tdbase
 * join` takes (src/tools/tdbase.cpp:482-549).  It exists to time the
 * reference's GPU path, compiled for sm_100a, beside this repository's on the
 * same tiles.  Prints the join's wall time on stderr as "join seconds: S".
 *
 * With TDP_REFGPU_RESULTS=PATH set, every result the join recorded is written
 * to PATH as one "qid rid" line per pair, read from each query object's result
 * list after the join.  The reference's --print_result prints only the
 * results that pass through HiMesh_Wrapper::report_result
 * (src/spatial/himesh_wrapper.cpp:195-202); within_chunking appends its
 * per-LOD results to the list directly (src/join/WithinJoin.cpp:781), so the
 * lists are the complete result set.
 *
 *   tdbase_ref_gpu --tile1 N.dt --tile2 V.dt -q within --within_dist 400 -g [--print_result]
 */
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

#include "SpatialJoin.h"
#include "mygpu.h"
#include "tile.h"

using namespace tdbase;

static double now_s() {
    timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec + 1e-6 * t.tv_usec;
}

int main(int argc, char** argv) {
    global_ctx = parse_args(argc, argv);
    geometry_computer* gc = new geometry_computer();
    if (global_ctx.use_gpu) {
        initialize();
        gc->init_gpus();
    }
    if (global_ctx.num_compute_thread > 0) gc->set_thread_num(global_ctx.num_compute_thread);
    std::vector<char> p1(global_ctx.tile1_path.begin(), global_ctx.tile1_path.end()), p2;
    p1.push_back(0);
    Tile* t1 = nullptr;
    Tile* t2 = nullptr;
    if (!global_ctx.tile2_path.empty()) {
        p2.assign(global_ctx.tile2_path.begin(), global_ctx.tile2_path.end());
        p2.push_back(0);
        t1 = new Tile(p1.data(), global_ctx.max_num_objects1, false);
        t2 = new Tile(p2.data(), global_ctx.max_num_objects2, false);
    } else {
        t1 = new Tile(p1.data(), LONG_MAX, false);
        t2 = t1;
    }
    const double l0 = now_s();
    t1->load();
    if (t2 != t1) t2->load();
    const double l1 = now_s();
    std::vector<std::pair<Tile*, Tile*>> pairs{{t1, t2}};
    SpatialJoin* joiner = new SpatialJoin(gc);
    const double j0 = now_s();
    joiner->join(pairs);
    const double j1 = now_s();
    std::fprintf(stderr, "load seconds: %f\njoin seconds: %f\n", l1 - l0, j1 - j0);
    if (const char* path = std::getenv("TDP_REFGPU_RESULTS")) {
        FILE* f = std::fopen(path, "w");
        if (!f) {
            std::fprintf(stderr, "cannot write %s\n", path);
            return 2;
        }
        size_t n = 0;
        for (size_t i = 0; i < t1->num_objects(); ++i) {
            HiMesh_Wrapper* w = t1->get_mesh_wrapper(i);
            for (HiMesh_Wrapper* r : w->results) {
                std::fprintf(f, "%ld %ld\n", (long)w->id, (long)r->id);
                ++n;
            }
        }
        std::fclose(f);
        std::fprintf(stderr, "results: %zu\n", n);
    }
    if (t2 != t1) delete t2;
    delete t1;
    delete joiner;
    delete gc;
    return 0;
}
