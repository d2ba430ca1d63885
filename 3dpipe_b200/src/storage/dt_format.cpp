// dt_format.cpp -- bounds-checked parser of the RAW tile format (see dt_format.h).
#include "storage/dt_format.h"

#include <cmath>
#include <cstring>

#include "tdp.h"

namespace tdp {

namespace {
template <typename T>
bool rd(const uint8_t* buf, size_t len, size_t& pos, T& v) {
    if (pos > len || len - pos < sizeof(T)) return false;
    std::memcpy(&v, buf + pos, sizeof(T));
    pos += sizeof(T);
    return true;
}
}  // namespace

size_t raw_object_bytes(uint32_t nvox, const uint32_t* counts) {
    size_t tris = 0;
    for (int l = 0; l < kNumLods; ++l)
        for (uint32_t v = 0; v < nvox; ++v) tris += counts[(size_t)l * nvox + v];
    return sizeof(size_t) + tris * 11 * sizeof(float) + sizeof(size_t) + kNumLods * 2 * sizeof(float) +
           (size_t)nvox * (9 * sizeof(float) + kNumLods * 2 * sizeof(size_t)) + 3 * sizeof(float);
}

int parse_raw_dt(const uint8_t* buf, size_t len, long max_objects, TileHost& T, std::string& err) {
    T = TileHost();
    if (!buf || len < 1) { err = "empty tile buffer"; return TDP_ERR_FORMAT; }
    if (buf[0] != kRawType) {
        err = "tile is not RAW (first byte " + std::to_string((int)buf[0]) + "); convert COMPRESSED tiles first";
        return TDP_ERR_FORMAT;
    }
    size_t pos = 1;
    T.obj_vox_off.push_back(0);
    while (pos < len && (max_objects <= 0 || T.n_obj < max_objects)) {
        const long id = T.n_obj;
        uint64_t data_size = 0;
        if (!rd(buf, len, pos, data_size)) { err = "truncated data_size of object " + std::to_string(id); return TDP_ERR_FORMAT; }
        const uint64_t data_off = pos;
        if (data_size > len - pos || data_size % 4) { err = "bad data_size of object " + std::to_string(id); return TDP_ERR_FORMAT; }
        pos += data_size;
        uint64_t vnum = 0;
        if (!rd(buf, len, pos, vnum) || vnum == 0 || vnum > (1u << 24)) {
            err = "bad voxel count of object " + std::to_string(id);
            return TDP_ERR_FORMAT;
        }
        float hd[kNumLods], phd[kNumLods];
        for (int l = 0; l < kNumLods; ++l)
            if (!rd(buf, len, pos, hd[l]) || !rd(buf, len, pos, phd[l])) { err = "truncated object hausdorff"; return TDP_ERR_FORMAT; }
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint64_t v = 0; v < vnum; ++v) {
            float b[9];
            for (int k = 0; k < 9; ++k)
                if (!rd(buf, len, pos, b[k])) { err = "truncated voxel record of object " + std::to_string(id); return TDP_ERR_FORMAT; }
            for (int k = 0; k < 3; ++k) {
                if (!(b[k] <= b[3 + k])) { err = "inverted voxel box in object " + std::to_string(id); return TDP_ERR_FORMAT; }
                lo[k] = std::fmin(lo[k], b[k]);
                hi[k] = std::fmax(hi[k], b[3 + k]);
            }
            T.vox_box.insert(T.vox_box.end(), b, b + 9);
            for (int l = 0; l < kNumLods; ++l) {
                uint64_t off = 0, cnt = 0;
                if (!rd(buf, len, pos, off) || !rd(buf, len, pos, cnt)) { err = "truncated voxel lod table"; return TDP_ERR_FORMAT; }
                if (cnt > (1u << 24) || off % 4 || off > data_size || cnt * 44 > data_size - off) {
                    err = "voxel lod range outside data block in object " + std::to_string(id);
                    return TDP_ERR_FORMAT;
                }
                T.vox_byte_off[l].push_back(data_off + off);
                T.vox_cnt[l].push_back((uint32_t)cnt);
                T.n_tris[l] += cnt;
            }
        }
        float xf[3];
        for (int k = 0; k < 3; ++k)
            if (!rd(buf, len, pos, xf[k])) { err = "truncated transform of object " + std::to_string(id); return TDP_ERR_FORMAT; }
        T.obj_data_off.push_back(data_off);
        T.obj_data_size.push_back(data_size);
        T.obj_vox_off.push_back((uint32_t)(T.obj_vox_off.back() + vnum));
        T.obj_box.insert(T.obj_box.end(), {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]});
        T.obj_xf.insert(T.obj_xf.end(), xf, xf + 3);
        T.obj_hd.insert(T.obj_hd.end(), hd, hd + kNumLods);
        T.obj_phd.insert(T.obj_phd.end(), phd, phd + kNumLods);
        T.n_obj++;
        if ((uint64_t)T.obj_vox_off.back() >= 0xffffffffull) { err = "too many voxels in tile"; return TDP_ERR_FORMAT; }
    }
    T.n_vox = T.obj_vox_off.back();
    if (T.n_obj == 0) { err = "tile holds no objects"; return TDP_ERR_FORMAT; }
    return TDP_OK;
}

}  // namespace tdp
