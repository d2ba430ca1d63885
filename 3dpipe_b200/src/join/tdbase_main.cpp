// tdbase_main.cpp -- the `tdbase join` command line on top of the C ABI.
//
// Same operator surface as the reference (src/tools/tdbase.cpp:482-549, options
// src/include/query_context.h:145-167):
//   tdbase join --tile1 P1 [--tile2 P2] -q nn|within [--knn K] [--within_dist T]
//               [-l LOD]... [--hausdorff_level 0|1|2] [--print_result] [-g]
//               [--max_objects1 N] [--max_objects2 N] [--form plain|tuned] [--device D]
// A missing --tile2 is a self-join (tdbase.cpp:511-514).  `--lod` is accepted as
// an alias of `-l/--lods` (the reference's README spelling).  -g, -t and --cn
// are accepted for compatibility; the join always runs on the GPU.
// Output: one "qid rid" line per result with --print_result
// (src/spatial/himesh_wrapper.cpp:198-200); timing and counts on stderr.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "tdp.h"

static bool read_file(const std::string& p, std::vector<unsigned char>& b) {
    std::ifstream f(p, std::ios::binary | std::ios::ate);
    if (!f) return false;
    std::streamsize n = f.tellg();
    f.seekg(0);
    b.resize((size_t)n);
    return (bool)f.read((char*)b.data(), n);
}

static int usage() {
    std::fprintf(stderr,
                 "usage: tdbase join --tile1 P1 [--tile2 P2] -q nn|within [--knn K] [--within_dist T]\n"
                 "                   [-l LOD]... [--hausdorff_level 0|1|2] [--print_result]\n"
                 "                   [--max_objects1 N] [--max_objects2 N] [--form plain|tuned] [--device D]\n");
    return 2;
}

int main(int argc, char** argv) {
    if (argc < 2 || std::strcmp(argv[1], "join") != 0) return usage();
    std::string t1, t2, q;
    tdp_join_params p;
    tdp_join_default_params(&p);
    bool print = false;
    long max1 = 0, max2 = 0;
    int device = 0;
    for (int i = 2; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&]() -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--tile1") t1 = val();
        else if (a == "--tile2") t2 = val();
        else if (a == "-q" || a == "--query") q = val();
        else if (a == "-k" || a == "--knn") p.knn = std::atoi(val());
        else if (a == "-w" || a == "--within_dist") p.within_dist = (float)std::atof(val());
        else if (a == "-l" || a == "--lods" || a == "--lod") {
            if (p.n_lods >= 8) { std::fprintf(stderr, "at most 8 LODs\n"); return 2; }
            p.lods[p.n_lods++] = std::atoi(val());
        } else if (a == "--hausdorff_level") p.hausdorff_level = std::atoi(val());
        else if (a == "--print_result") print = true;
        else if (a == "--max_objects1") max1 = std::atol(val());
        else if (a == "--max_objects2") max2 = std::atol(val());
        else if (a == "--form") {
            std::string f = val();
            if (f == "plain") p.form = TDP_FORM_PLAIN;
            else if (f == "tuned") p.form = TDP_FORM_TUNED;
            else { std::fprintf(stderr, "unknown form %s (plain or tuned)\n", f.c_str()); return 2; }
        } else if (a == "--device") device = std::atoi(val());
        else if (a == "-g" || a == "--gpu" || a == "--aabb") {
        } else if (a == "-t" || a == "--threads" || a == "--cn" || a == "-v" || a == "--verbose") val();
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return usage(); }
    }
    if (t1.empty() || q.empty()) return usage();
    if (q == "nn") p.query = TDP_QUERY_NN;
    else if (q == "within") p.query = TDP_QUERY_WITHIN;
    else if (q == "intersect") p.query = TDP_QUERY_INTERSECT;
    else { std::fprintf(stderr, "error query type: %s\n", q.c_str()); return 2; }

    auto t0 = std::chrono::steady_clock::now();
    std::vector<unsigned char> b1, b2;
    if (!read_file(t1, b1)) { std::fprintf(stderr, "%s does not exist\n", t1.c_str()); return 1; }
    if (!t2.empty() && !read_file(t2, b2)) { std::fprintf(stderr, "%s does not exist\n", t2.c_str()); return 1; }
    tdp_ctx* ctx = nullptr;
    int rc = tdp_ctx_create(device, 0, 0, &ctx);
    if (rc) { std::fprintf(stderr, "cannot open device %d (status %d)\n", device, rc); return 1; }
    tdp_tile *T1 = nullptr, *T2 = nullptr;
    if ((rc = tdp_tile_upload(ctx, b1.data(), b1.size(), max1, &T1)) ||
        (!t2.empty() && (rc = tdp_tile_upload(ctx, b2.data(), b2.size(), max2, &T2)))) {
        std::fprintf(stderr, "tile load failed: %s\n", tdp_last_error(ctx));
        tdp_ctx_destroy(ctx);
        return 1;
    }
    auto t1c = std::chrono::steady_clock::now();
    tdp_result* r = nullptr;
    if ((rc = tdp_join(ctx, T1, T2, &p, &r))) {
        std::fprintf(stderr, "join failed: %s\n", tdp_last_error(ctx));
        tdp_ctx_destroy(ctx);
        return 1;
    }
    auto t2c = std::chrono::steady_clock::now();
    long n = 0;
    tdp_result_count(r, &n);
    std::vector<int> qs(n), rs(n);
    tdp_result_copy(r, qs.data(), rs.data(), nullptr);
    if (print)
        for (long i = 0; i < n; ++i) std::printf("%d %d\n", qs[i], rs[i]);
    tdp_stats st;
    tdp_last_stats(ctx, &st);
    tdp_tile_info info;
    tdp_tile_get_info(T1, &info);
    std::fprintf(stderr, "load:\t%f\njoin:\t%f\n", std::chrono::duration<double>(t1c - t0).count(),
                 std::chrono::duration<double>(t2c - t1c).count());
    std::fprintf(stderr, "refine_ms:\t%f\nfilter_ms:\t%f\ntri_pairs:\t%.0f\n", st.refine_ms, st.filter_ms, st.tri_pairs);
    std::fprintf(stderr, "#objects:\t%ld\n results:%ld(\t%.3f)\n", info.n_objects, n,
                 info.n_objects ? (double)n / info.n_objects : 0.0);
    tdp_result_free(r);
    tdp_tile_free(ctx, T1);
    if (T2) tdp_tile_free(ctx, T2);
    tdp_ctx_destroy(ctx);
    return 0;
}
