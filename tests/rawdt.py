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
