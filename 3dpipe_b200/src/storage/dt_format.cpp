// dt_format.cpp -- bounds-checked parser of the RAW tile format (see dt_format.h).
#include "storage/dt_format.h"
#include "storage/host_pool.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>

#include "tdp.h"

#if defined(__SSE__)
#include <xmmintrin.h>
#endif

namespace tdp {

namespace {

struct HostBlockCache {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;  // capacity -> freed block
    std::unordered_map<void*, size_t> cap;     // capacity of every block the cache made
    size_t cached = 0;                         // bytes in free_blocks
};

// never destroyed: tiles may release their arrays during static destruction
HostBlockCache& host_cache() {
    static HostBlockCache* c = new HostBlockCache();
    return *c;
}

// free cached blocks (smallest first) until at most `keep` bytes stay; the
// caller holds the lock
void host_cache_shrink(HostBlockCache& c, size_t keep) {
    while (c.cached > keep && !c.free_blocks.empty()) {
        auto it = c.free_blocks.begin();
        c.cached -= it->first;
        c.cap.erase(it->second);
        std::free(it->second);
        c.free_blocks.erase(it);
    }
}

}  // namespace

void* host_block_get(size_t bytes) {
    HostBlockCache& c = host_cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.free_blocks.lower_bound(bytes);
    if (it != c.free_blocks.end() && it->first - bytes <= bytes / 8) {
        void* p = it->second;
        c.cached -= it->first;
        c.free_blocks.erase(it);
        return p;
    }
    void* p = std::malloc(bytes);
    if (!p) {
        host_cache_shrink(c, 0);
        p = std::malloc(bytes);
        if (!p) throw std::bad_alloc();
    }
    c.cap[p] = bytes;
    return p;
}

void host_block_put(void* p, size_t bytes) {
    if (!p) return;
    HostBlockCache& c = host_cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.cap.find(p);
    const size_t cap = it != c.cap.end() ? it->second : bytes;
    if (cap > kHostCacheMax) {
        if (it != c.cap.end()) c.cap.erase(it);
        std::free(p);
        return;
    }
    host_cache_shrink(c, kHostCacheMax - cap);
    c.free_blocks.emplace(cap, p);
    c.cached += cap;
}

size_t host_cache_bytes() {
    HostBlockCache& c = host_cache();
    std::lock_guard<std::mutex> g(c.mu);
    return c.cached;
}

void host_cache_trim() {
    HostBlockCache& c = host_cache();
    std::lock_guard<std::mutex> g(c.mu);
    host_cache_shrink(c, 0);
}

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

namespace {

// object o's data block holds, LOD by LOD and voxel by voxel, each voxel's
// triangles then their bounds, with nothing in between
bool object_canonical(const TileHost& T, long o, uint32_t v0, uint32_t v1) {
    uint64_t expect = T.obj_data_off[o];
    for (int l = 0; l < kNumLods; ++l)
        for (uint32_t v = v0; v < v1; ++v) {
            if (T.vox_byte_off[l][v] != expect) return false;
            expect += 44ull * T.vox_cnt[l][v];
        }
    return true;
}

// One object after another: the reference reader's order.  Used as is for the
// exact first error of a malformed tile.
int parse_sequential(const uint8_t* buf, size_t len, long max_objects, TileHost& T, std::string& err) {
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
    for (long o = 0; o < T.n_obj && T.first_noncanonical < 0; ++o)
        if (!object_canonical(T, o, T.obj_vox_off[o], T.obj_vox_off[o + 1])) T.first_noncanonical = o;
    T.chunk_vox = {0, (uint64_t)T.n_vox};
    T.chunk_tris.assign(1, {});
    for (int l = 0; l < kNumLods; ++l) T.chunk_tris[0][l] = T.n_tris[l];
    return TDP_OK;
}

}  // namespace

namespace {

using Rec = RawRec;

// One voxel record in the device layout (low xyz, 0, high xyz, 0, core xyz,
// 0).  The records are read again only by the copy to the device, so on x86
// a 16-byte aligned destination is written with non-temporal stores, which
// skip reading each line into the cache first (a sixth of the parse of a
// 100k-object tile); store_fence() makes them visible before the copy.
inline void store_record(float* d, const float* b, bool stream) {
#if defined(__SSE__)
    if (stream) {
        _mm_stream_ps(d, _mm_setr_ps(b[0], b[1], b[2], 0.f));
        _mm_stream_ps(d + 4, _mm_setr_ps(b[3], b[4], b[5], 0.f));
        _mm_stream_ps(d + 8, _mm_setr_ps(b[6], b[7], b[8], 0.f));
        return;
    }
#else
    (void)stream;
#endif
    const float rec[12] = {b[0], b[1], b[2], 0.f, b[3], b[4], b[5], 0.f, b[6], b[7], b[8], 0.f};
    std::memcpy(d, rec, sizeof(rec));
}

inline void store_fence() {
#if defined(__SSE__)
    _mm_sfence();
#endif
}
constexpr size_t kVoxBytes = 9 * sizeof(float) + kNumLods * 2 * sizeof(uint64_t);

// the record of the object whose first byte is at pos; false on a structural
// problem (the sequential parser then reports it)
inline bool walk_one(const uint8_t* buf, size_t len, size_t& pos, Rec& r) {
    uint64_t data_size = 0, vnum = 0;
    if (!rd(buf, len, pos, data_size) || data_size > len - pos || data_size % 4) return false;
    r.data_off = pos;
    r.data_size = data_size;
    pos += data_size;
    if (!rd(buf, len, pos, vnum) || vnum == 0 || vnum > (1u << 24)) return false;
    const uint64_t rec = 2 * kNumLods * sizeof(float) + vnum * kVoxBytes + 3 * sizeof(float);
    if (rec > len - pos) return false;
    r.meta = pos;
    r.vnum = vnum;
    pos += rec;
    return true;
}

// up to `limit` records from pos into out (count in n, pos past the last);
// false on a structural problem.  Every object's position depends on the
// sizes read at the previous one, so this is a chain of dependent loads: the
// headers of the next few objects are prefetched at the last record's stride
// (a wrong guess only wastes a prefetch).
bool walk_chain(const uint8_t* buf, size_t len, size_t& pos, long limit, Rec* out, long& n) {
    constexpr int kAhead = 8;
    uint64_t stride = 0, last_ds = 0;
    n = 0;
    while (pos < len && n < limit) {
        if (stride)
            for (int k = 1; k <= kAhead; ++k) {
                const uint64_t q = pos + k * stride;
                if (q + 8 + last_ds + 8 > len) break;
                __builtin_prefetch(buf + q);
                __builtin_prefetch(buf + q + 8 + last_ds);
            }
        const size_t start = pos;
        if (!walk_one(buf, len, pos, out[n])) return false;
        stride = pos - start;
        last_ds = out[n].data_size;
        ++n;
    }
    return true;
}

}  // namespace

// Two passes: a walk over the size fields finds every object's record (a
// structural problem hands the tile to the sequential parser, which reports
// the first error in file order); then the objects' voxel tables are read in
// parallel into arrays sized from the walk.  Content errors are reported for
// the lowest object that has one, the error the sequential parser would meet
// first, with the same message.
bool raw_first_record(const uint8_t* buf, size_t len, RawRec& r, uint64_t& stride) {
    if (!buf || len < 2 || buf[0] != kRawType) return false;
    size_t p = 1;
    if (!walk_one(buf, len, p, r)) return false;
    stride = p - 1;
    return true;
}

bool walk_raw_dt(const uint8_t* buf, size_t len, long max_objects, HostVec<RawRec>& recs) {
    recs.clear();
    if (!buf || len < 1 || buf[0] != kRawType) return false;
    size_t pos = 1;
    // Objects of one tile are mostly the same size (instances of one mesh):
    // with many objects, threads walk chunks from guessed starts at the
    // first object's stride.  A chunk counts only when the walk before it
    // ends exactly on its start, so what is kept is what the serial walk
    // would find; the walk continues serially from the last verified
    // position (a wrong guess, a structural problem, the tile's end).
    if (max_objects <= 0) {
        size_t p1 = 1;
        Rec r0;
        const long hw = (long)host_threads();
        if (walk_one(buf, len, p1, r0)) {
            const uint64_t stride = p1 - 1;
            const long n_est = (long)((len - 1) / stride);
            const long nt = std::min(hw, n_est / 4096);
            if (nt >= 2) {
                const long per = (n_est + nt - 1) / nt;
                recs.resize((size_t)(nt * per));
                std::vector<long> got(nt, 0);
                std::vector<size_t> end(nt, 0);
                std::vector<char> clean(nt, 0);
                host_for(nt, [&](long k) {
                    size_t q = 1 + (size_t)(k * per) * stride;
                    if (q >= len) return;
                    long c = 0;
                    clean[k] = walk_chain(buf, len, q, per, &recs[(size_t)(k * per)], c);
                    got[k] = c;
                    end[k] = q;
                });
                long kept = 0;
                for (long k = 0; k < nt; ++k) {
                    if (!clean[k] || 1 + (size_t)(k * per) * stride != pos) break;
                    kept += got[k];
                    pos = end[k];
                    if (got[k] != per) break;
                }
                recs.resize((size_t)kept);
            }
        }
    }
    {
        size_t q = pos;
        long c = 0;
        const long room = max_objects <= 0 ? -1 : max_objects;
        while (q < len && (room < 0 || (long)recs.size() < room)) {
            // serial walk in blocks (the block's records land in place)
            const long block = room < 0 ? 65536 : std::min<long>(65536, room - (long)recs.size());
            const size_t at = recs.size();
            recs.resize(at + (size_t)block);
            c = 0;
            const bool ok = walk_chain(buf, len, q, block, &recs[at], c);
            recs.resize(at + (size_t)c);
            if (!ok) return false;
        }
    }
    return true;
}

int parse_raw_dt(const uint8_t* buf, size_t len, long max_objects, TileHost& T, std::string& err,
                 const VoxSink& sink) {
    T = TileHost();
    if (!buf || len < 1) { err = "empty tile buffer"; return TDP_ERR_FORMAT; }
    if (buf[0] != kRawType) return parse_sequential(buf, len, max_objects, T, err);
    HostVec<Rec> recs;
    if (!walk_raw_dt(buf, len, max_objects, recs)) return parse_sequential(buf, len, max_objects, T, err);
    uint64_t nvox = 0;
    for (const Rec& r : recs) nvox += r.vnum;
    if (nvox >= 0xffffffffull) return parse_sequential(buf, len, max_objects, T, err);
    const long n = (long)recs.size();
    if (n == 0) { err = "tile holds no objects"; return TDP_ERR_FORMAT; }
    T.n_obj = n;
    T.n_vox = (long)nvox;
    T.obj_vox_off.resize(n + 1);
    T.obj_vox_off[0] = 0;
    for (long o = 0; o < n; ++o) T.obj_vox_off[o + 1] = T.obj_vox_off[o] + (uint32_t)recs[o].vnum;
    T.obj_data_off.resize(n);
    T.obj_data_size.resize(n);
    T.obj_box.resize(6 * n);
    T.obj_xf.resize(3 * n);
    T.obj_hd.resize((size_t)kNumLods * n);
    T.obj_phd.resize((size_t)kNumLods * n);
    float* vrec = sink ? sink((long)nvox, n) : nullptr;  // device-layout voxel records
    const bool stream = vrec && ((uintptr_t)vrec & 15) == 0;
    if (!vrec) T.vox_box.resize(9 * nvox);
    for (int l = 0; l < kNumLods; ++l) {
        T.vox_byte_off[l].resize(nvox);
        T.vox_cnt[l].resize(nvox);
    }
    // chunks of whole objects with about equal voxel counts (a vessel tile
    // has few objects of many voxels each)
    const int nt = (int)std::max<long>(1, std::min<long>({(long)host_threads(), (long)(nvox / 2048), n}));
    std::vector<long> first(nt + 1, n);
    for (int k = 0; k < nt; ++k)
        first[k] = std::lower_bound(T.obj_vox_off.begin(), T.obj_vox_off.begin() + n, (uint32_t)(nvox * k / nt)) -
                   T.obj_vox_off.begin();
    std::vector<long> bad(nt, -1);
    std::vector<std::string> msg(nt);
    std::vector<std::array<uint64_t, kNumLods>> tris(nt);
    std::vector<long> noncanon(nt, -1);
    auto work = [&](int k) {
        long nc = -1;  // this chunk's lowest non-canonical object, in a register
        struct FlushNc {
            long& dst;
            const long& src;
            ~FlushNc() { dst = src; }
        } flush_nc{noncanon[k], nc};
        uint64_t nt_l[kNumLods] = {0, 0, 0, 0, 0};  // per thread, in registers (no shared cache line)
        struct Flush {
            std::array<uint64_t, kNumLods>& dst;
            const uint64_t* src;
            ~Flush() { for (int l = 0; l < kNumLods; ++l) dst[l] = src[l]; }
        } flush{tris[k], nt_l};
        const long o_end = first[k + 1];
        for (long o = first[k]; o < o_end; ++o) {
            const Rec& r = recs[o];
            if (o + 4 < o_end) {  // the metadata of a later object, ahead of its turn
                const Rec& f = recs[o + 4];
                const uint64_t bytes = 2 * kNumLods * sizeof(float) + f.vnum * kVoxBytes;
                for (uint64_t b = 0; b < bytes; b += 64) __builtin_prefetch(buf + f.meta + b);
            }
            const uint8_t* p = buf + r.meta;
            float hp[2 * kNumLods];
            std::memcpy(hp, p, sizeof(hp));
            p += sizeof(hp);
            for (int l = 0; l < kNumLods; ++l) {
                T.obj_hd[(size_t)o * kNumLods + l] = hp[2 * l];
                T.obj_phd[(size_t)o * kNumLods + l] = hp[2 * l + 1];
            }
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            const uint32_t v0 = T.obj_vox_off[o];
            for (uint64_t v = 0; v < r.vnum; ++v) {
                float box[9];
                float* b = vrec ? box : &T.vox_box[9 * (size_t)(v0 + v)];
                std::memcpy(b, p, 9 * sizeof(float));
                if (vrec) store_record(vrec + 12 * (size_t)(v0 + v), b, stream);
                p += 9 * sizeof(float);
                for (int c = 0; c < 3; ++c) {
                    if (!(b[c] <= b[3 + c])) {
                        bad[k] = o;
                        msg[k] = "inverted voxel box in object " + std::to_string(o);
                        return;
                    }
                    lo[c] = std::fmin(lo[c], b[c]);
                    hi[c] = std::fmax(hi[c], b[3 + c]);
                }
                uint64_t oc[2 * kNumLods];
                std::memcpy(oc, p, sizeof(oc));
                p += sizeof(oc);
                for (int l = 0; l < kNumLods; ++l) {
                    const uint64_t off = oc[2 * l], cnt = oc[2 * l + 1];
                    if (cnt > (1u << 24) || off % 4 || off > r.data_size || cnt * 44 > r.data_size - off) {
                        bad[k] = o;
                        msg[k] = "voxel lod range outside data block in object " + std::to_string(o);
                        return;
                    }
                    T.vox_byte_off[l][v0 + v] = r.data_off + off;
                    T.vox_cnt[l][v0 + v] = (uint32_t)cnt;
                    nt_l[l] += cnt;
                }
            }
            std::memcpy(&T.obj_xf[3 * o], p, 3 * sizeof(float));
            T.obj_data_off[o] = r.data_off;
            if (nc < 0 && !object_canonical(T, o, v0, v0 + (uint32_t)r.vnum)) nc = o;
            T.obj_data_size[o] = r.data_size;
            float* ob = &T.obj_box[6 * o];
            ob[0] = lo[0]; ob[1] = lo[1]; ob[2] = lo[2];
            ob[3] = hi[0]; ob[4] = hi[1]; ob[5] = hi[2];
        }
        store_fence();
    };
    host_for(nt, [&](long k) { work((int)k); });
    for (int k = 0; k < nt; ++k)
        if (bad[k] >= 0) {  // chunks are in object order: the first failing chunk holds the lowest object
            err = msg[k];
            T = TileHost();
            return TDP_ERR_FORMAT;
        }
    for (int k = 0; k < nt; ++k)
        for (int l = 0; l < kNumLods; ++l) T.n_tris[l] += tris[k][l];
    for (int k = 0; k < nt && T.first_noncanonical < 0; ++k) T.first_noncanonical = noncanon[k];
    T.chunk_vox.resize(nt + 1);
    for (int k = 0; k <= nt; ++k) T.chunk_vox[k] = T.obj_vox_off[first[k]];
    T.chunk_tris = std::move(tris);
    return TDP_OK;
}

void vtri_prefix(const TileHost& T, uint32_t* const out[kNumLods], uint32_t* const stage[kNumLods]) {
    const long nk = (long)T.chunk_tris.size();
    const long tasks = nk * kNumLods;
    auto run = [&](long task) {
        const int l = (int)(task % kNumLods);
        const long k = task / kNumLods;
        uint64_t base = 0;
        for (long j = 0; j < k; ++j) base += T.chunk_tris[j][l];
        const uint32_t* cnt = T.vox_cnt[l].data();
        uint32_t* o = out[l];
        uint32_t* st = stage[l];
        uint32_t run_sum = (uint32_t)base;
        const uint64_t vb = T.chunk_vox[k], ve = T.chunk_vox[k + 1];
        if (k == 0) {
            o[0] = 0;
            if (st) st[0] = 0;
        }
        if (st) {
            for (uint64_t v = vb; v < ve; ++v) {
                run_sum += cnt[v];
                o[v + 1] = run_sum;
                st[v + 1] = run_sum;
            }
        } else {
            for (uint64_t v = vb; v < ve; ++v) {
                run_sum += cnt[v];
                o[v + 1] = run_sum;
            }
        }
    };
    host_for(tasks, [&](long t) { run(t); });
}

}  // namespace tdp

extern "C" int tdp_raw_check(const void* raw, size_t len, long* n_objects, long* n_voxels, char* err, size_t err_len) {
    tdp::TileHost T;
    std::string e;
    const int rc = tdp::parse_raw_dt((const uint8_t*)raw, len, 0, T, e);
    if (n_objects) *n_objects = rc == TDP_OK ? T.n_obj : 0;
    if (n_voxels) *n_voxels = rc == TDP_OK ? T.n_vox : 0;
    if (err && err_len) {
        const size_t k = std::min(err_len - 1, e.size());
        std::memcpy(err, e.data(), k);
        err[k] = 0;
    }
    return rc;
}

extern "C" size_t tdp_host_cache_bytes(void) { return tdp::host_cache_bytes(); }
extern "C" void tdp_host_cache_trim(void) { tdp::host_cache_trim(); }
