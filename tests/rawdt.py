"""Independent numpy reader of the reference's RAW .dt tile format (test infrastructure).

Restates HiMesh_Wrapper(char*, id, RAW) (reference src/spatial/himesh_wrapper.cpp:17-83)
and Tile::load (src/storage/tile_IO.cpp:13-49) so tests can check the C++
parser, the generator and the CUDA path against a second reading of the bytes.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

LODS = (20, 40, 60, 80, 100)


@dataclass
class Obj:
    voxels: np.ndarray           # [nv, 9] low xyz, high xyz, core xyz
    tris: list                   # per lod: list per voxel of float32 [n, 9]
    hds: list                    # per lod: list per voxel of float32 [n, 2]
    hausdorff: np.ndarray        # [5]
    proxyhausdorff: np.ndarray   # [5]
    transform: np.ndarray        # [3]

    @property
    def box(self):
        return np.concatenate([self.voxels[:, :3].min(0), self.voxels[:, 3:6].max(0)])

    def lod_tris(self, li):
        return np.concatenate(self.tris[li]) if self.tris[li] else np.zeros((0, 9), np.float32)


def read_tile(buf, max_objects=None):
    b = bytes(buf) if not isinstance(buf, (bytes, bytearray)) else buf
    assert b[0] == 1, "not a RAW tile"
    pos = 1
    objs = []
    while pos < len(b) and (max_objects is None or len(objs) < max_objects):
        (data_size,) = struct.unpack_from("<Q", b, pos)
        pos += 8
        data = pos
        pos += data_size
        (vnum,) = struct.unpack_from("<Q", b, pos)
        pos += 8
        hp = np.frombuffer(b, np.float32, 10, pos).reshape(5, 2)
        pos += 40
        vox = np.zeros((vnum, 9), np.float32)
        offc = np.zeros((vnum, 5, 2), np.int64)
        for v in range(vnum):
            vox[v] = np.frombuffer(b, np.float32, 9, pos)
            pos += 36
            offc[v] = np.frombuffer(b, np.uint64, 10, pos).reshape(5, 2).astype(np.int64)
            pos += 80
        xf = np.frombuffer(b, np.float32, 3, pos).copy()
        pos += 12
        tris, hds = [], []
        for li in range(5):
            tl, hl = [], []
            for v in range(vnum):
                off, n = offc[v, li]
                tl.append(np.frombuffer(b, np.float32, 9 * n, data + off).reshape(n, 9))
                hl.append(np.frombuffer(b, np.float32, 2 * n, data + off + 36 * n).reshape(n, 2))
            tris.append(tl)
            hds.append(hl)
        objs.append(Obj(vox, tris, hds, hp[:, 0].copy(), hp[:, 1].copy(), xf))
    return objs


def write_tile(objects, lod_order=(0, 1, 2, 3, 4)):
    """RAW tile bytes (uint8 array) from objects given as [lod][voxel] -> float32
    array [n, 9]; bounds written as zeros, voxel boxes from the triangles, core =
    the first vertex.  lod_order: the order in which the LOD blocks are laid out
    in each object's data block (the writer's order is 20, 40, ..., 100)."""
    out = bytearray([1])
    for obj in objects:
        nv = len(obj[4])
        data = bytearray()
        offc = np.zeros((nv, 5, 2), np.uint64)
        for li in lod_order:
            for v in range(nv):
                t = np.asarray(obj[li][v], np.float32).reshape(-1, 9)
                offc[v, li] = (len(data), len(t))
                data += t.tobytes() + np.zeros((len(t), 2), np.float32).tobytes()
        out += struct.pack("<Q", len(data)) + data + struct.pack("<Q", nv) + np.zeros(10, np.float32).tobytes()
        for v in range(nv):
            pts = np.concatenate([np.asarray(obj[li][v], np.float32).reshape(-1, 3) for li in range(5)])
            lo, hi = pts.min(0), pts.max(0)
            out += np.concatenate([lo, hi, pts[0]]).astype(np.float32).tobytes() + offc[v].tobytes()
        out += np.zeros(3, np.float32).tobytes()
    return np.frombuffer(bytes(out), np.uint8).copy()


def first_problem(b, pos=1, obj=0, resume=None):
    """Restatement of a sequential read of RAW tile bytes (the order and the
    messages of the reader the C++ parser reports for, after the reference's
    HiMesh_Wrapper(char*, id, RAW), src/spatial/himesh_wrapper.cpp:17-83),
    starting at byte `pos` with object id `obj`.  `resume` maps byte offsets
    to the ids of records known to be intact from there to the end: reaching
    one ends the read.  Returns ("error", message) or ("ok", objects read,
    voxels read, id of the intact record reached or None)."""
    mv = memoryview(b)
    n = len(mv)
    nvox = 0
    start = obj

    def u64(p):
        return struct.unpack_from("<Q", mv, p)[0] if p + 8 <= n else None

    while pos < n:
        if resume is not None and pos in resume:
            return ("ok", obj - start, nvox, resume[pos])
        ds = u64(pos)
        if ds is None:
            return ("error", f"truncated data_size of object {obj}")
        pos += 8
        if ds > n - pos or ds % 4:
            return ("error", f"bad data_size of object {obj}")
        pos += ds
        vn = u64(pos)
        if vn is None or vn == 0 or vn > (1 << 24):
            return ("error", f"bad voxel count of object {obj}")
        pos += 8
        if pos + 40 > n:
            return ("error", "truncated object hausdorff")
        pos += 40
        for _ in range(vn):
            if pos + 36 > n:
                return ("error", f"truncated voxel record of object {obj}")
            box = struct.unpack_from("<9f", mv, pos)
            pos += 36
            for k in range(3):
                if not (box[k] <= box[3 + k]):
                    return ("error", f"inverted voxel box in object {obj}")
            for _ in range(5):
                if pos + 16 > n:
                    return ("error", "truncated voxel lod table")
                off, cnt = struct.unpack_from("<QQ", mv, pos)
                pos += 16
                if cnt > (1 << 24) or off % 4 or off > ds or cnt * 44 > ds - off:
                    return ("error", f"voxel lod range outside data block in object {obj}")
        if pos + 12 > n:
            return ("error", f"truncated transform of object {obj}")
        pos += 12
        nvox += vn
        obj += 1
    if obj == 0:
        return ("error", "tile holds no objects")
    return ("ok", obj - start, nvox, None)
