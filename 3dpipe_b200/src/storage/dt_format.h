// dt_format.h -- the reference's RAW tile format (`.dt`, Decoding_Type RAW = 1).
//
// Layout (written by Tile::dump_raw_stream, reference src/storage/tile_IO.cpp:79-172;
// read by HiMesh_Wrapper(char*, id, RAW), src/spatial/himesh_wrapper.cpp:17-83, and
// Tile::load, src/storage/tile_IO.cpp:13-49):
//
//   uint8   type                                   (1 = RAW)
//   per object, in file order (object id = position):
//     size_t  data_size
//     data block: for lod in 20,40,60,80,100: for each voxel:
//                 float tri[9*n]  then  float hd[2*n]   (hd = proxy, hausdorff)
//     size_t  vnum
//     for lod in 20..100:  float hausdorff, float proxyhausdorff     (object level)
//     for each voxel: float low[3], high[3], core[3];
//                     for lod in 20..100: size_t offset (bytes, into the data block), size_t count
//     float   transform[3]
//
// The object's box is the union of its voxel boxes (himesh_wrapper.cpp:40, :80).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <memory>
#include <utility>
#include <vector>

namespace tdp {

constexpr int kNumLods = 5;
constexpr int kLods[kNumLods] = {20, 40, 60, 80, 100};
constexpr uint8_t kRawType = 1;

inline int lod_index(int lod) {
    for (int i = 0; i < kNumLods; ++i)
        if (kLods[i] == lod) return i;
    return -1;
}

// Large host arrays (kHostBlockMin bytes and up) are recycled through a
// process-wide cache of freed blocks.  A block fresh from the system arrives
// as untouched pages, every first touch of one costs a page fault, and handing
// it back costs an munmap: for a 100k-object tile that was about half of the
// parse.  The cache keeps at most kHostCacheMax bytes of freed blocks and
// serves a request from a cached block at most 1/8 larger.
constexpr size_t kHostBlockMin = size_t(1) << 20;
constexpr size_t kHostCacheMax = size_t(4) << 30;
void* host_block_get(size_t bytes);  // throws std::bad_alloc
void host_block_put(void* p, size_t bytes);
size_t host_cache_bytes();           // freed bytes held by the cache now
void host_cache_trim();              // free every cached block

// An allocator whose resize() leaves new elements of plain types
// uninitialised: the parser writes every element from its own threads, so a
// tile's arrays are touched first there (in parallel) instead of being
// zeroed by one thread beforehand.  Large arrays come from the host block
// cache.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    using value_type = T;
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    T* allocate(size_t n) {
        if (n * sizeof(T) >= kHostBlockMin) return static_cast<T*>(host_block_get(n * sizeof(T)));
        return std::allocator<T>::allocate(n);
    }
    void deallocate(T* p, size_t n) {
        if (n * sizeof(T) >= kHostBlockMin) host_block_put(p, n * sizeof(T));
        else std::allocator<T>::deallocate(p, n);
    }
    template <typename U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <typename T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

// Host-side view of a parsed RAW tile.  Offsets point into the caller's byte buffer.
struct TileHost {
    long n_obj = 0;
    long n_vox = 0;
    HostVec<uint64_t> obj_data_off;     // byte offset of each object's data block
    HostVec<uint64_t> obj_data_size;
    HostVec<uint32_t> obj_vox_off;      // [n_obj+1]
    HostVec<float> obj_box;             // 6 per object: low xyz, high xyz
    HostVec<float> obj_xf;              // 3 per object
    HostVec<float> obj_hd;              // kNumLods per object (hausdorff)
    HostVec<float> obj_phd;             // kNumLods per object (proxy hausdorff)
    HostVec<float> vox_box;             // 9 per voxel: low xyz, high xyz, core xyz
    HostVec<uint64_t> vox_byte_off[kNumLods];  // absolute byte offset of the voxel's triangles
    HostVec<uint32_t> vox_cnt[kNumLods];
    uint64_t n_tris[kNumLods] = {0, 0, 0, 0, 0};
    // lowest object whose data block does not hold, LOD by LOD and voxel by
    // voxel, each voxel's triangles then their bounds with nothing in between
    // (the layout the reference's writer produces, src/storage/tile_IO.cpp:79-172); -1
    // when every object does
    long first_noncanonical = -1;
    // the parser's chunks: chunk k holds voxels [chunk_vox[k], chunk_vox[k + 1])
    // and chunk_tris[k][l] triangles at LOD index l
    std::vector<uint64_t> chunk_vox;
    std::vector<std::array<uint64_t, kNumLods>> chunk_tris;
};

// out[l][v] = triangles at LOD index l in voxels [0, v), for v in [0, n_vox]
// (out[l] holds n_vox + 1 entries), written also to stage[l] where that is
// not null: host threads over (LOD, parser chunk) tasks, each chunk starting
// from the triangle totals of the chunks before it.
void vtri_prefix(const TileHost& T, uint32_t* const out[kNumLods], uint32_t* const stage[kNumLods]);

// Optional destination of the voxel records in the device layout, 12 floats
// per voxel (low xyz, 0, high xyz, 0, core xyz, 0): called once with the
// voxel and object counts before the voxel tables are read.  When it returns
// a pointer, the records go there and vox_box stays empty; when it returns
// nullptr (or the tile takes the sequential parser), vox_box is filled.
using VoxSink = std::function<float*(long n_vox, long n_obj)>;

// One object's record as the walk over the size fields finds it: where its
// data block starts and how long it is, where its metadata start (the
// per-LOD object Hausdorff values, after vnum) and how many voxels it has.
struct RawRec {
    uint64_t data_off, data_size, meta, vnum;
};

// The walk alone (the first pass of parse_raw_dt): the records of at most
// max_objects objects (<= 0: all).  Returns false on a structural problem
// (parse_raw_dt then reports it) or when the tile does not start with the RAW
// type byte; the voxel tables are not read.
bool walk_raw_dt(const uint8_t* buf, size_t len, long max_objects, HostVec<RawRec>& recs);

// The record of the first object and its length in bytes (the stride), or
// false when the first record is not well formed.
bool raw_first_record(const uint8_t* buf, size_t len, RawRec& r, uint64_t& stride);

// Parse `len` bytes; at most max_objects objects (<= 0: all).  Returns 0 or a
// TDP_ERR_* code with a message in `err`.
int parse_raw_dt(const uint8_t* buf, size_t len, long max_objects, TileHost& out, std::string& err,
                 const VoxSink& sink = {});

// Size in bytes of one object's record given its voxel count and per-(lod,voxel)
// triangle counts (counts[l * nvox + v]).
size_t raw_object_bytes(uint32_t nvox, const uint32_t* counts);

}  // namespace tdp
