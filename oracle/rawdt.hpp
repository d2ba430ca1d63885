// oracle/rawdt.hpp -- TEST INFRASTRUCTURE ONLY.
// Minimal reader of the reference's RAW .dt tile format for the CPU checkers,
// written independently of the product's parser
// (format: reference src/storage/tile_IO.cpp:79-172, src/spatial/himesh_wrapper.cpp:48-83).
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace oracle {

struct RVoxel {
    float low[3], high[3], core[3];
    uint64_t off[5], cnt[5];  // byte offset into the object's data block, triangle count
};

struct RObject {
    const uint8_t* data = nullptr;  // start of the data block
    float hd[5], phd[5];
    std::vector<RVoxel> vox;
    float transform[3];
    float box[6];
    // copies (aligned) of a voxel's triangles / hausdorff at LOD index li
    void tris(int v, int li, std::vector<float>& t, std::vector<float>& h) const {
        const RVoxel& x = vox[v];
        t.resize(9 * x.cnt[li]);
        h.resize(2 * x.cnt[li]);
        if (x.cnt[li]) {
            std::memcpy(t.data(), data + x.off[li], 36 * x.cnt[li]);
            std::memcpy(h.data(), data + x.off[li] + 36 * x.cnt[li], 8 * x.cnt[li]);
        }
    }
};

inline std::vector<RObject> read_tile(const uint8_t* b, size_t len) {
    if (len < 1 || b[0] != 1) throw std::runtime_error("not a RAW tile");
    std::vector<RObject> objs;
    size_t pos = 1;
    auto get = [&](void* dst, size_t n) {
        if (pos + n > len) throw std::runtime_error("truncated tile");
        std::memcpy(dst, b + pos, n);
        pos += n;
    };
    while (pos < len) {
        RObject o;
        uint64_t ds, vn;
        get(&ds, 8);
        o.data = b + pos;
        pos += ds;
        get(&vn, 8);
        for (int l = 0; l < 5; ++l) {
            get(&o.hd[l], 4);
            get(&o.phd[l], 4);
        }
        o.vox.resize(vn);
        for (auto& v : o.vox) {
            get(v.low, 12);
            get(v.high, 12);
            get(v.core, 12);
            for (int l = 0; l < 5; ++l) {
                get(&v.off[l], 8);
                get(&v.cnt[l], 8);
            }
        }
        get(o.transform, 12);
        for (int k = 0; k < 3; ++k) {
            o.box[k] = INFINITY;
            o.box[3 + k] = -INFINITY;
        }
        for (auto& v : o.vox)
            for (int k = 0; k < 3; ++k) {
                o.box[k] = std::fmin(o.box[k], v.low[k]);
                o.box[3 + k] = std::fmax(o.box[3 + k], v.high[k]);
            }
        objs.push_back(std::move(o));
    }
    return objs;
}

}  // namespace oracle
