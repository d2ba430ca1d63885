"""Python binding of the tdp C ABI (include/tdp.h) over ctypes.

This is the host-side mirror of the reference's `tdbase join` operator surface
and of its refine seam (geometry_computer::get_distance, reference
src/geometry/geometry_computer.cpp:86-222).  It loads the in-tree
3dpipe_b200/libtdp.so and fails loudly when that library is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libtdp.so"

TDP_OK = 0
ERRORS = {1: "TDP_ERR_ARG", 2: "TDP_ERR_CUDA", 3: "TDP_ERR_NOMEM", 4: "TDP_ERR_FORMAT",
          5: "TDP_ERR_TIMEOUT", 6: "TDP_ERR_STATE", 7: "TDP_ERR_NODEV"}
FORM_PLAIN, FORM_TUNED = 0, 1
QUERY_NN, QUERY_WITHIN, QUERY_INTERSECT = 1, 2, 3

# Every symbol include/tdp.h declares; tests check the library exports them all.
EXPORTED = [
    "tdp_ctx_create", "tdp_ctx_destroy", "tdp_last_error", "tdp_ctx_memory", "tdp_last_stats",
    "tdp_refine_batch", "tdp_gen_default_params", "tdp_gen_tiles",
]


class TdpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [("refine_ms", C.c_double), ("filter_ms", C.c_double), ("total_ms", C.c_double),
                ("full_evals", C.c_ulonglong), ("tri_pairs", C.c_double), ("refine_items", C.c_long),
                ("refine_launches", C.c_long), ("recheck_pairs", C.c_long), ("filter_pairs", C.c_long),
                ("filter_voxel_pairs", C.c_double), ("kernel_launches", C.c_long),
                ("candidates_ms", C.c_double), ("lod_ms", C.c_double), ("host_syncs", C.c_long),
                ("exact_ms", C.c_double), ("exact_items", C.c_long), ("exact_f64_items", C.c_long),
                ("fp32_max_rel_err", C.c_double), ("fetch_bytes", C.c_double), ("lod_graph", C.c_long),
                ("refine_ms_lod", C.c_double * 5), ("exact_phase_ms", C.c_double * 4),
                ("exact_full_evals", C.c_ulonglong), ("candidates_on_device", C.c_long),
                ("candidate_redone", C.c_long), ("exact_dropped_items", C.c_long),
                ("exact_below_items", C.c_long)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["refine_ms_lod"] = list(self.refine_ms_lod)
        d["exact_phase_ms"] = list(self.exact_phase_ms)
        return d


_lib = None


def lib() -> C.CDLL:
    """Load libtdp.so (built in-tree by 3dpipe_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python 3dpipe_b200/build.py` "
                           "(the CUDA extension is required; there is no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    L.tdp_ctx_create.argtypes = [C.c_int, C.c_size_t, C.c_uint, C.POINTER(P)]
    L.tdp_ctx_destroy.argtypes = [P]
    L.tdp_last_error.argtypes = [P]
    L.tdp_last_error.restype = C.c_char_p
    L.tdp_ctx_memory.argtypes = [P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.tdp_last_stats.argtypes = [P, C.POINTER(Stats)]
    L.tdp_refine_batch.argtypes = [P, P, P, C.c_size_t, P, C.c_uint32, C.c_int, P]
    L.tdp_gen_default_params.argtypes = [P]
    L.tdp_gen_default_params.restype = None
    L.tdp_gen_tiles.argtypes = [P, P, C.c_size_t, P, P, C.c_size_t, P, C.c_char_p, C.c_size_t]
    _bind_join(L)
    _lib = L
    return L


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class GenParams(C.Structure):
    _fields_ = [("n_vessels", C.c_int), ("nuclei_per_vessel", C.c_int), ("seed", C.c_uint64),
                ("voxel_size", C.c_int), ("nucleus_subdiv", C.c_int), ("tube_sides", C.c_int),
                ("tube_rings", C.c_int), ("threads", C.c_int), ("grid", C.c_float),
                ("shell_min", C.c_float), ("shell_max", C.c_float), ("nuclei_begin", C.c_long),
                ("nuclei_end", C.c_long)]


def gen_tiles(n_vessels: int = 10, nuclei_per_vessel: int = 20, seed: int = 20260001, out=None, only=None, **kw):
    """Generate (nuclei_tile_bytes, vessel_tile_bytes) as uint8 arrays in RAW .dt format.

    `out`, if given, is a callable (nbytes) -> writable uint8 array (for example a
    pinned buffer); otherwise numpy arrays are allocated.  only="nuclei" or
    "vessels" writes just that tile (the other is returned as None)."""
    L = lib()
    p = GenParams()
    L.tdp_gen_default_params(C.byref(p))
    p.n_vessels, p.nuclei_per_vessel, p.seed = n_vessels, nuclei_per_vessel, seed
    for k, v in kw.items():
        setattr(p, k, v)
    nl, vl = C.c_size_t(), C.c_size_t()
    err = C.create_string_buffer(512)
    rc = L.tdp_gen_tiles(C.byref(p), None, 0, C.byref(nl), None, 0, C.byref(vl), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode())
    if only not in (None, "nuclei", "vessels"):
        raise ValueError("only must be None, 'nuclei' or 'vessels'")
    alloc = out or (lambda n: np.empty(n, np.uint8))
    nb = alloc(nl.value) if only != "vessels" else None
    vb = alloc(vl.value) if only != "nuclei" else None
    rc = L.tdp_gen_tiles(C.byref(p), _ptr(nb), 0 if nb is None else nb.size, C.byref(nl), _ptr(vb),
                         0 if vb is None else vb.size, C.byref(vl), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode())
    return (None if nb is None else nb[:nl.value]), (None if vb is None else vb[:vl.value])


class Context:
    """A device context: stream, memory budget, scratch buffers."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, flags: int = 0):
        L = lib()
        h = C.c_void_p()
        rc = L.tdp_ctx_create(device, budget_bytes, flags, C.byref(h))
        if rc != TDP_OK:
            raise TdpError(rc, "tdp_ctx_create failed (device %d)" % device)
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().tdp_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int):
        if rc != TDP_OK:
            raise TdpError(rc, lib().tdp_last_error(self._h).decode())

    def stats(self) -> dict:
        s = Stats()
        self.check(lib().tdp_last_stats(self._h, C.byref(s)))
        return s.as_dict()

    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        L = lib()
        L.tdp_ctx_stream.argtypes = [C.c_void_p]
        L.tdp_ctx_stream.restype = C.c_void_p
        return L.tdp_ctx_stream(self._h) or 0

    def set_lod_graph(self, mode: int):
        """How the tuned LOD loop launches: LOD_GRAPH_OFF (directly), LOD_GRAPH_AUTO
        (default: a CUDA graph captured on the second join with the same launch
        arguments, replayed after that) or LOD_GRAPH_ALWAYS."""
        L = lib()
        L.tdp_set_lod_graph.argtypes = [C.c_void_p, C.c_int]
        self.check(L.tdp_set_lod_graph(self._h, int(mode)))

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        self.check(lib().tdp_ctx_memory(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def refine_batch(self, data: np.ndarray, hausdorff: np.ndarray | None, offset_size: np.ndarray,
                     form: int = FORM_PLAIN) -> np.ndarray:
        """Batched refine with the reference's seam layout.

        data: float32 [E, 9]; hausdorff: float32 [E, 2] or None;
        offset_size: uint64 [P, 4] rows (off1, n1, off2, n2).
        Returns float32 [P, 3]: (distance, min_dist, max_dist)."""
        data = np.ascontiguousarray(data, np.float32).reshape(-1, 9)
        hd = None if hausdorff is None else np.ascontiguousarray(hausdorff, np.float32).reshape(-1, 2)
        osz = np.ascontiguousarray(offset_size, np.uint64).reshape(-1, 4)
        out = np.empty((osz.shape[0], 3), np.float32)
        self.check(lib().tdp_refine_batch(self._h, _ptr(data), _ptr(hd), data.shape[0], _ptr(osz),
                                          osz.shape[0], form, _ptr(out)))
        return out


class TileInfo(C.Structure):
    _fields_ = [("n_objects", C.c_long), ("n_voxels", C.c_long), ("n_tris", C.c_long * 5),
                ("device_bytes", C.c_size_t), ("h2d_bytes", C.c_size_t), ("attached", C.c_int),
                ("parse_ms", C.c_double), ("alloc_ms", C.c_double), ("load_ms", C.c_double),
                ("meta_ms", C.c_double)]


class JoinParams(C.Structure):
    _fields_ = [("query", C.c_int), ("knn", C.c_int), ("within_dist", C.c_float), ("lods", C.c_int * 8),
                ("n_lods", C.c_int), ("hausdorff_level", C.c_int), ("form", C.c_int),
                ("exact_distances", C.c_int), ("obj_knn", C.c_void_p), ("obj_within", C.c_void_p),
                ("query_begin", C.c_long), ("query_end", C.c_long)]


def _bind_join(L):
    P = C.c_void_p
    L.tdp_tile_upload.argtypes = [P, P, C.c_size_t, C.c_long, C.POINTER(P)]
    L.tdp_tile_attach.argtypes = [P, P, C.c_size_t, C.c_long, C.POINTER(P)]
    L.tdp_tile_free.argtypes = [P, P]
    L.tdp_tile_get_info.argtypes = [P, C.POINTER(TileInfo)]
    L.tdp_candidates.argtypes = [P, P, C.c_long, P, P, C.c_long, C.c_int, C.c_int, C.c_int, C.c_float, P, P, C.c_long]
    L.tdp_candidates.restype = C.c_long
    L.tdp_join_default_params.argtypes = [C.POINTER(JoinParams)]
    L.tdp_join_default_params.restype = None
    L.tdp_join.argtypes = [P, P, P, C.POINTER(JoinParams), C.POINTER(P)]
    L.tdp_result_count.argtypes = [P, C.POINTER(C.c_long)]
    L.tdp_result_copy.argtypes = [P, P, P, P]
    L.tdp_result_free.argtypes = [P]


EXPORTED += ["tdp_tile_upload", "tdp_tile_free", "tdp_tile_get_info", "tdp_candidates",
             "tdp_join_default_params", "tdp_join", "tdp_result_count", "tdp_result_copy", "tdp_result_free"]


class Tile:
    """A RAW .dt tile resident in HBM (Tile::load + decode to every LOD), or,
    with attach=True, attached: `raw` stays in page-locked host memory (it must
    be registered, e.g. with cudaHostRegister, or come from pinned_empty, and it
    must outlive the tile) and joins fetch the voxels they refine
    (tdp_tile_attach)."""

    def __init__(self, ctx: "Context", raw: np.ndarray, max_objects: int = 0, attach: bool = False):
        if attach:
            if not (isinstance(raw, np.ndarray) and raw.dtype == np.uint8 and raw.flags.c_contiguous):
                raise ValueError("attach needs the tile's own contiguous uint8 buffer (page-locked)")
        else:
            raw = np.ascontiguousarray(raw, np.uint8)
        h = C.c_void_p()
        fn = lib().tdp_tile_attach if attach else lib().tdp_tile_upload
        ctx.check(fn(ctx.handle, _ptr(raw), raw.size, max_objects, C.byref(h)))
        self._ctx, self._h = ctx, h
        self._raw = raw if attach else None  # the host bytes an attached tile reads

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        i = TileInfo()
        lib().tdp_tile_get_info(self._h, C.byref(i))
        return {"n_objects": i.n_objects, "n_voxels": i.n_voxels, "n_tris": list(i.n_tris),
                "device_bytes": i.device_bytes, "h2d_bytes": i.h2d_bytes, "attached": bool(i.attached),
                "parse_ms": i.parse_ms, "alloc_ms": i.alloc_ms, "load_ms": i.load_ms, "meta_ms": i.meta_ms}

    def free(self):
        if getattr(self, "_h", None):
            lib().tdp_tile_free(self._ctx.handle, self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def candidates(box1, xf1, box2, xf2, self_join=False, knn=0, within=0.0, intersect=False):
    """Object candidates (CSR offsets, ids); knn > 0 selects the kNN query,
    intersect the strict box-overlap query."""
    L = lib()
    box1 = np.ascontiguousarray(box1, np.float32).reshape(-1, 6)
    box2 = np.ascontiguousarray(box2, np.float32).reshape(-1, 6)
    xf1 = np.ascontiguousarray(xf1, np.float32).reshape(-1, 3)
    xf2 = np.ascontiguousarray(xf2, np.float32).reshape(-1, 3)
    off = np.zeros(len(box1) + 1, np.int64)
    mode = 2 if intersect else int(knn > 0)
    n = L.tdp_candidates(_ptr(box1), _ptr(xf1), len(box1), _ptr(box2), _ptr(xf2), len(box2), int(self_join),
                         mode, max(knn, 1), float(within), _ptr(off), None, 0)
    ids = np.zeros(max(-n, 1), np.int32)
    n = L.tdp_candidates(_ptr(box1), _ptr(xf1), len(box1), _ptr(box2), _ptr(xf2), len(box2), int(self_join),
                         mode, max(knn, 1), float(within), _ptr(off), _ptr(ids), ids.size)
    if n < 0:
        raise TdpError(1, "tdp_candidates failed")
    return off, ids[:n]


def _join_params(query, knn, within, lods, hausdorff_level, form) -> JoinParams:
    p = JoinParams()
    lib().tdp_join_default_params(C.byref(p))
    if query not in ("nn", "within", "intersect"):
        raise ValueError("query must be nn, within or intersect")
    p.query = {"nn": QUERY_NN, "within": QUERY_WITHIN, "intersect": QUERY_INTERSECT}[query]
    p.knn, p.within_dist, p.hausdorff_level, p.form = knn, within, hausdorff_level, form
    if lods:
        p.n_lods = len(lods)
        for i, l in enumerate(lods):
            p.lods[i] = l
    return p


def _join(self, tile1: Tile, tile2: Tile | None, query: str = "nn", knn: int = 1, within: float = 1000.0,
          lods=None, hausdorff_level: int = 2, form: int = FORM_TUNED, exact_distances: bool = False,
          obj_knn=None, obj_within=None, query_range=None):
    """tdbase join on resident tiles; returns (query_ids, result_ids, dist) sorted by (query, result).

    dist is float32 (each pair's upper bound when decided) unless
    exact_distances is set: then float64 exact LOD-100 distances.  obj_knn /
    obj_within (one entry per tile-1 object) give every query object its own
    query: K > 0 for kNN, 0 for within at obj_within[i].  query_range = (b, e)
    joins only tile-1 objects [b, e) (one shard of a split join; ids stay
    tile-1 ids)."""
    L = lib()
    p = _join_params(query, knn, within, lods, hausdorff_level, form)
    p.exact_distances = int(bool(exact_distances))
    if query_range is not None:
        p.query_begin, p.query_end = int(query_range[0]), int(query_range[1])
    keep = []
    if obj_knn is not None:
        ok = np.ascontiguousarray(obj_knn, np.int32)
        ow = np.ascontiguousarray(np.zeros(len(ok)) if obj_within is None else obj_within, np.float32)
        if ok.shape != ow.shape:
            raise ValueError("obj_knn and obj_within need one entry per query object")
        keep = [ok, ow]
        p.obj_knn, p.obj_within = ok.ctypes.data, ow.ctypes.data
    r = C.c_void_p()
    self.check(L.tdp_join(self._h, tile1.handle, None if tile2 is None else tile2.handle, C.byref(p), C.byref(r)))
    try:
        n = C.c_long()
        L.tdp_result_count(r, C.byref(n))
        q = np.empty(n.value, np.int32)
        t = np.empty(n.value, np.int32)
        d = np.empty(n.value, np.float32)
        L.tdp_result_copy(r, _ptr(q), _ptr(t), _ptr(d))
        if exact_distances:
            d = np.empty(n.value, np.float64)
            L.tdp_result_copy_f64.argtypes = [C.c_void_p, C.c_void_p]
            rc = L.tdp_result_copy_f64(r, _ptr(d))
            if rc != TDP_OK:
                raise TdpError(rc, "exact distances missing")
    finally:
        L.tdp_result_free(r)
    return q, t, d


Context.join = _join


EXPORTED += ["tdp_fp32_peak", "tdp_refine_batch_noalloc", "tdp_tile_candidates", "tdp_ctx_stream",
             "tdp_refine_config_count", "tdp_refine_config_info", "tdp_set_refine_config", "tdp_get_refine_config",
             "tdp_autotune", "tdp_result_copy_f64", "tdp_server_default_params", "tdp_server_create",
             "tdp_server_submit", "tdp_server_wait", "tdp_server_get_stats", "tdp_server_destroy",
             "tdp_join_chunked", "tdp_set_lod_graph"]

LOD_GRAPH_OFF, LOD_GRAPH_AUTO, LOD_GRAPH_ALWAYS = 0, 1, 2

EXPORTED += ["tdp_tile_compute_bounds", "tdp_raw_compute_bounds", "tdp_tile_attach", "tdp_host_alloc",
             "tdp_host_free", "tdp_raw_check", "tdp_get_refine_config_lod", "tdp_host_cache_bytes",
             "tdp_host_cache_trim", "tdp_partition_queries", "tdp_raw_partition"]


def partition_queries(raw1, raw2=None, n_shards=2, knn=0, within=0.0, intersect=False):
    """Split the query objects of RAW tile raw1 (raw2 None: a self-join) into
    n_shards contiguous ranges of about equal estimated work (tdp_raw_partition,
    host only).  Returns (bounds[n_shards + 1], work[n_shards])."""
    L = lib()
    L.tdp_raw_partition.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_float,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    r1 = np.ascontiguousarray(raw1, np.uint8)
    r2 = None if raw2 is None else np.ascontiguousarray(raw2, np.uint8)
    bounds = np.zeros(int(n_shards) + 1, np.int64)
    work = np.zeros(int(n_shards), np.float64)
    err = C.create_string_buffer(512)
    mode = 2 if intersect else int(knn > 0)
    rc = L.tdp_raw_partition(_ptr(r1), r1.size, None if r2 is None else _ptr(r2), 0 if r2 is None else r2.size,
                             mode, max(int(knn), 1), float(within), int(n_shards), _ptr(bounds), _ptr(work), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode() or "tdp_raw_partition failed")
    return bounds, work

CTX_POISON = 1  # tdp_ctx_create flag: unfetched records of attached tiles read as NaN


def raw_check(raw):
    """Validate RAW tile bytes on the host: (n_objects, n_voxels), or TdpError
    (TDP_ERR_FORMAT) naming the first problem in file order."""
    L = lib()
    L.tdp_raw_check.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_long), C.POINTER(C.c_long), C.c_char_p,
                                C.c_size_t]
    raw = np.ascontiguousarray(raw, np.uint8)
    no, nv = C.c_long(), C.c_long()
    err = C.create_string_buffer(512)
    rc = L.tdp_raw_check(_ptr(raw), raw.size, C.byref(no), C.byref(nv), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode())
    return no.value, nv.value


def host_cache_bytes() -> int:
    """Freed host bytes the parser's process-wide block cache holds now."""
    L = lib()
    L.tdp_host_cache_bytes.restype = C.c_size_t
    L.tdp_host_cache_bytes.argtypes = []
    return int(L.tdp_host_cache_bytes())


def host_cache_trim() -> None:
    """Hand every block of the parser's host block cache back to the system."""
    L = lib()
    L.tdp_host_cache_trim.restype = None
    L.tdp_host_cache_trim.argtypes = []
    L.tdp_host_cache_trim()


def pinned_empty(nbytes: int) -> np.ndarray:
    """A uint8 array in page-locked host memory (tdp_host_alloc), freed when the
    array is collected: the buffer to read a tile into before attaching it."""
    import weakref
    L = lib()
    L.tdp_host_alloc.argtypes = [C.c_size_t, C.POINTER(C.c_void_p)]
    L.tdp_host_free.argtypes = [C.c_void_p]
    p = C.c_void_p()
    rc = L.tdp_host_alloc(int(nbytes), C.byref(p))
    if rc != TDP_OK:
        raise TdpError(rc, f"tdp_host_alloc({nbytes}) failed")
    buf = (C.c_uint8 * int(nbytes)).from_address(p.value)
    arr = np.frombuffer(buf, np.uint8)
    weakref.finalize(buf, L.tdp_host_free, p.value)
    return arr


def pinned_copy(raw: np.ndarray) -> np.ndarray:
    """`raw` copied into page-locked host memory (see pinned_empty)."""
    out = pinned_empty(raw.size)
    out[:] = np.asarray(raw, np.uint8).ravel()
    return out


class BoundsInfo(C.Structure):
    _fields_ = [("ms", C.c_double), ("objects", C.c_long), ("triangles", C.c_long), ("facet_queries", C.c_long),
                ("pieces", C.c_long), ("dist_evals", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _compute_bounds(self, tile: "Tile") -> dict:
    """Recompute the per-triangle (proxy, hausdorff) bounds and the object-level
    values of a resident tile on the GPU, in place; returns the kernel stats."""
    L = lib()
    L.tdp_tile_compute_bounds.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(BoundsInfo)]
    info = BoundsInfo()
    self.check(L.tdp_tile_compute_bounds(self._h, tile.handle, C.byref(info)))
    return info.as_dict()


def _raw_compute_bounds(self, raw, out=None):
    """RAW tile bytes -> (the same bytes with GPU-computed bounds, stats).  `out`
    (uint8, raw's size) receives the result; it may be `raw` itself."""
    L = lib()
    L.tdp_raw_compute_bounds.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.POINTER(BoundsInfo)]
    src = np.ascontiguousarray(raw, np.uint8)
    dst = np.empty_like(src) if out is None else out
    if dst.nbytes != src.nbytes or not dst.flags.c_contiguous:
        raise ValueError("out must be a contiguous buffer of the tile's size")
    info = BoundsInfo()
    self.check(L.tdp_raw_compute_bounds(self._h, _ptr(src), src.nbytes, _ptr(dst), C.byref(info)))
    return dst, info.as_dict()


Context.compute_bounds = _compute_bounds
Context.raw_compute_bounds = _raw_compute_bounds


class ChunkedInfo(C.Structure):
    _fields_ = [("chunks", C.c_long), ("splits", C.c_long), ("h2d_bytes", C.c_double), ("tri_pairs", C.c_double),
                ("join_ms", C.c_double), ("device_peak_bytes", C.c_double)]


def _join_chunked(self, raw1: np.ndarray, raw2: np.ndarray, chunk_objects: int, query: str = "nn", knn: int = 1,
                  within: float = 1000.0, lods=None, hausdorff_level: int = 2, form: int = FORM_TUNED):
    """A join of host RAW tiles in chunks of query objects (tdp_join_chunked);
    returns (q, t, d, info) with global ids, equal to the whole join."""
    L = lib()
    raw1 = np.ascontiguousarray(raw1, np.uint8)
    raw2 = np.ascontiguousarray(raw2, np.uint8)
    p = _join_params(query, knn, within, lods, hausdorff_level, form)
    r = C.c_void_p()
    inf = ChunkedInfo()
    L.tdp_join_chunked.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                   C.POINTER(JoinParams), C.c_long, C.POINTER(ChunkedInfo), C.POINTER(C.c_void_p)]
    self.check(L.tdp_join_chunked(self._h, _ptr(raw1), raw1.size, _ptr(raw2), raw2.size, C.byref(p),
                                  int(chunk_objects), C.byref(inf), C.byref(r)))
    try:
        n = C.c_long()
        L.tdp_result_count(r, C.byref(n))
        q = np.empty(n.value, np.int32)
        t = np.empty(n.value, np.int32)
        d = np.empty(n.value, np.float32)
        L.tdp_result_copy(r, _ptr(q), _ptr(t), _ptr(d))
    finally:
        L.tdp_result_free(r)
    return q, t, d, {k: getattr(inf, k) for k, _ in inf._fields_}


Context.join_chunked = _join_chunked


def raw_object_offsets(raw: np.ndarray) -> np.ndarray:
    """Byte offset of every object record of a RAW .dt tile, plus the end:
    [n+1] int64.  Record layout (reference src/storage/tile_IO.cpp:79-172):
    u64 data_size, data, u64 vnum, 5 x (hausdorff, proxy) floats, vnum x
    (9 floats + 5 x (u64 offset, u64 count)), 3 floats of transform."""
    import struct
    mv = memoryview(np.ascontiguousarray(raw, np.uint8))
    off, n = 1, len(mv)
    out = [off]
    while off < n:
        (ds,) = struct.unpack_from("<Q", mv, off)
        p = off + 8 + ds
        (vn,) = struct.unpack_from("<Q", mv, p)
        off = p + 8 + 40 + vn * 116 + 12
        if off > n:
            raise ValueError("truncated RAW tile")
        out.append(off)
    return np.asarray(out, np.int64)


def raw_slice(raw: np.ndarray, offsets: np.ndarray, b: int, e: int) -> np.ndarray:
    """A RAW .dt tile holding objects [b, e) of `raw` (its type byte first)."""
    return np.concatenate([raw[:1], raw[offsets[b]:offsets[e]]])


class ServerParams(C.Structure):
    _fields_ = [("arena_objects", C.c_long), ("arena_voxels", C.c_long), ("arena_tris", C.c_long),
                ("max_request_bytes", C.c_size_t), ("lods", C.c_int * 8), ("n_lods", C.c_int),
                ("hausdorff_level", C.c_int), ("form", C.c_int), ("big_request_ms", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("latency_ms", C.c_double), ("batch", C.c_long),
                ("batch_requests", C.c_int), ("status", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("batches", C.c_long), ("requests", C.c_long), ("failed", C.c_long), ("busy_ms", C.c_double),
                ("upload_ms", C.c_double), ("upload_bytes", C.c_double), ("fetch_bytes", C.c_double),
                ("split_batches", C.c_long)]


class Server:
    """Continuous-batching request loop over a resident tile 2 (tdp_server_*).

    submit() takes a RAW .dt tile of query objects plus its own query and
    returns at once; wait() returns that request's (query ids, result ids,
    distances) with the request's own object ids, and its latency record.
    The context belongs to the server until close()."""

    def __init__(self, ctx: "Context", tile2: "Tile", **params):
        L = lib()
        P = C.c_void_p
        L.tdp_server_default_params.argtypes = [C.POINTER(ServerParams)]
        L.tdp_server_default_params.restype = None
        L.tdp_server_create.argtypes = [P, P, C.POINTER(ServerParams), C.POINTER(P)]
        L.tdp_server_submit.argtypes = [P, P, C.c_size_t, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_uint64)]
        L.tdp_server_wait.argtypes = [P, C.c_uint64, C.c_int, C.POINTER(P), C.POINTER(RequestInfo)]
        L.tdp_server_get_stats.argtypes = [P, C.POINTER(ServerStats)]
        L.tdp_server_destroy.argtypes = [P]
        p = ServerParams()
        L.tdp_server_default_params(C.byref(p))
        for k, v in params.items():
            if k == "lods":
                p.n_lods = len(v)
                for i, l in enumerate(v):
                    p.lods[i] = l
            else:
                setattr(p, k, v)
        h = C.c_void_p()
        ctx.check(L.tdp_server_create(ctx.handle, tile2.handle, C.byref(p), C.byref(h)))
        self._ctx, self._tile2, self._h = ctx, tile2, h
        self._bufs = {}

    def submit(self, raw: np.ndarray, query: str = "nn", knn: int = 1, within: float = 0.0) -> int:
        raw = np.ascontiguousarray(raw, np.uint8)
        rid = C.c_uint64()
        rc = lib().tdp_server_submit(self._h, _ptr(raw), raw.size, QUERY_NN if query == "nn" else QUERY_WITHIN,
                                     int(knn), float(within), C.byref(rid))
        if rc != TDP_OK:
            raise TdpError(rc, "request rejected")
        self._bufs[rid.value] = raw  # the bytes must live until the request completes
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """(q, t, d, info) of a finished request; None if timeout_ms ran out."""
        L = lib()
        r = C.c_void_p()
        info = RequestInfo()
        rc = L.tdp_server_wait(self._h, rid, int(timeout_ms), C.byref(r), C.byref(info))
        if rc == 5:  # TDP_ERR_TIMEOUT
            return None
        self._bufs.pop(rid, None)
        if rc != TDP_OK:
            raise TdpError(rc, "request failed")
        try:
            n = C.c_long()
            L.tdp_result_count(r, C.byref(n))
            q = np.empty(n.value, np.int32)
            t = np.empty(n.value, np.int32)
            d = np.empty(n.value, np.float32)
            L.tdp_result_copy(r, _ptr(q), _ptr(t), _ptr(d))
        finally:
            L.tdp_result_free(r)
        return q, t, d, {"queue_ms": info.queue_ms, "latency_ms": info.latency_ms, "batch": info.batch,
                         "batch_requests": info.batch_requests}

    def stats(self) -> dict:
        s = ServerStats()
        lib().tdp_server_get_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().tdp_server_destroy(self._h)
            self._h = None
            self._bufs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refine_configs():
    """[(chunk_a, ctas_per_sm)] of the tuned refine kernel's configurations."""
    L = lib()
    out = []
    for i in range(L.tdp_refine_config_count()):
        a, c = C.c_int(), C.c_int()
        L.tdp_refine_config_info(i, C.byref(a), C.byref(c))
        out.append((a.value, c.value))
    return out


def _set_refine_config(self, cfg: int):
    lib().tdp_set_refine_config.argtypes = [C.c_void_p, C.c_int]
    self.check(lib().tdp_set_refine_config(self._h, int(cfg)))


def _get_refine_config(self) -> int:
    v = C.c_int()
    lib().tdp_get_refine_config.argtypes = [C.c_void_p, C.c_void_p]
    self.check(lib().tdp_get_refine_config(self._h, C.byref(v)))
    return v.value


def _autotune(self, tile1, tile2=None, query="within", knn=1, within=1000.0, lods=None, hausdorff_level=2):
    """Time every tuned-refine configuration on this join and keep the fastest;
    returns (best index, [refine ms per configuration])."""
    L = lib()
    p = _join_params(query, knn, within, lods, hausdorff_level, FORM_TUNED)
    n = L.tdp_refine_config_count()
    ms = (C.c_double * n)()
    best = C.c_int()
    L.tdp_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(JoinParams), C.c_void_p, C.c_void_p]
    self.check(L.tdp_autotune(self._h, tile1.handle, None if tile2 is None else tile2.handle, C.byref(p), ms,
                              C.byref(best)))
    return best.value, list(ms)


def _refine_configs_by_lod(self) -> dict:
    """{LOD: configuration} the tuned form uses at each LOD."""
    L = lib()
    L.tdp_get_refine_config_lod.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    out = {}
    for lod in (20, 40, 60, 80, 100):
        v = C.c_int()
        self.check(L.tdp_get_refine_config_lod(self._h, lod, C.byref(v)))
        out[lod] = v.value
    return out


Context.set_refine_config = _set_refine_config
Context.refine_config = _get_refine_config
Context.refine_configs_by_lod = _refine_configs_by_lod
Context.autotune = _autotune


def tile_candidates(ctx, tile1, tile2=None, knn=0, within=0.0):
    """Object candidates computed on the GPU from resident tiles: (CSR offsets, ids)."""
    L = lib()
    L.tdp_tile_candidates.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p,
                                      C.c_void_p, C.c_long]
    L.tdp_tile_candidates.restype = C.c_long
    n1 = tile1.info()["n_objects"]
    off = np.zeros(n1 + 1, np.int64)
    t2 = None if tile2 is None else tile2.handle
    n = L.tdp_tile_candidates(ctx.handle, tile1.handle, t2, int(knn > 0), max(knn, 1), float(within), _ptr(off), None, 0)
    if n == -(2 ** 63):
        raise TdpError(2, L.tdp_last_error(ctx.handle).decode())
    ids = np.zeros(max(-n, 1), np.int32)
    n = L.tdp_tile_candidates(ctx.handle, tile1.handle, t2, int(knn > 0), max(knn, 1), float(within), _ptr(off),
                              _ptr(ids), ids.size)
    if n < 0:
        raise TdpError(2, L.tdp_last_error(ctx.handle).decode())
    return off, ids[:n]


def _fp32_peak(self) -> float:
    """Measured FP32 FMA throughput (TFLOP/s) of this context's GPU."""
    v = C.c_double()
    lib().tdp_fp32_peak.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    self.check(lib().tdp_fp32_peak(self._h, C.byref(v)))
    return v.value


Context.fp32_peak = _fp32_peak


# ---- LOD preparation (GPU) ------------------------------------------------
EXPORTED += ["tdp_raw_prep_bound", "tdp_raw_from_meshes", "tdp_gen_meshes"]


class PrepInfo(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("decimate_ms", C.c_double), ("voxel_ms", C.c_double),
                ("write_ms", C.c_double), ("bounds_ms", C.c_double), ("n_objects", C.c_long),
                ("n_triangles", C.c_long * 5), ("n_voxels", C.c_long), ("batches", C.c_long)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["n_triangles"] = list(self.n_triangles)
        return d


def _mesh_arrays(vertices, vert_off, faces, face_off):
    V = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    F = np.ascontiguousarray(faces, np.uint32).reshape(-1)
    vo = np.ascontiguousarray(vert_off, np.int64)
    fo = np.ascontiguousarray(face_off, np.int64)
    if vo.size != fo.size or vo.size < 1:
        raise ValueError("vert_off and face_off need n_objects + 1 entries each")
    if vo[-1] * 3 > V.size or fo[-1] * 3 > F.size:
        raise ValueError("offsets run past the vertex or facet arrays")
    return V, vo, F, fo


def raw_prep_bound(face_off, voxel_size=100):
    """Bytes that always hold tdp_raw_from_meshes' tile of these objects."""
    L = lib()
    L.tdp_raw_prep_bound.argtypes = [C.c_void_p, C.c_long, C.c_int, C.POINTER(C.c_size_t)]
    fo = np.ascontiguousarray(face_off, np.int64)
    n = C.c_size_t()
    rc = L.tdp_raw_prep_bound(_ptr(fo), fo.size - 1, voxel_size, C.byref(n))
    if rc != TDP_OK:
        raise TdpError(rc, "tdp_raw_prep_bound: bad arguments")
    return n.value


def _raw_from_meshes(self, vertices, vert_off, faces, face_off, voxel_size=100, out=None):
    """LOD-100 meshes -> (RAW tile bytes, prep stats), every step on the GPU.
    Object o: vertices[vert_off[o]:vert_off[o+1]] (x, y, z) and facets
    faces[face_off[o]:face_off[o+1]] (indices local to the object).  `out`
    (a writable uint8 buffer of at least raw_prep_bound bytes) receives it."""
    L = lib()
    L.tdp_raw_from_meshes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_int,
                                      C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(PrepInfo)]
    V, vo, F, fo = _mesh_arrays(vertices, vert_off, faces, face_off)
    cap = raw_prep_bound(fo, voxel_size)
    buf = np.empty(cap, np.uint8) if out is None else out
    if buf.nbytes < cap or not buf.flags.c_contiguous:
        raise ValueError("out must be a contiguous buffer of at least raw_prep_bound bytes")
    n = C.c_size_t()
    info = PrepInfo()
    self.check(L.tdp_raw_from_meshes(self._h, _ptr(V), _ptr(vo), _ptr(F), _ptr(fo), fo.size - 1, voxel_size,
                                     _ptr(buf), buf.nbytes, C.byref(n), C.byref(info)))
    return buf[:n.value], info.as_dict()


Context.raw_from_meshes = _raw_from_meshes


def gen_meshes(n_vessels=10, nuclei_per_vessel=20, seed=20260001, which="nuclei", **kw):
    """The LOD-100 meshes of the generator's objects (the same vertices its
    tiles hold): (vertices[nv, 3] float32, vert_off, faces[nf, 3] uint32, face_off)."""
    L = lib()
    L.tdp_gen_meshes.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t,
                                 C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_long),
                                 C.c_char_p, C.c_size_t]
    p = GenParams()
    L.tdp_gen_default_params(C.byref(p))
    p.n_vessels, p.nuclei_per_vessel, p.seed = n_vessels, nuclei_per_vessel, seed
    for k, v in kw.items():
        setattr(p, k, v)
    w = {"nuclei": 0, "vessels": 1}[which]
    nv, nf, no = C.c_size_t(), C.c_size_t(), C.c_long()
    err = C.create_string_buffer(512)
    rc = L.tdp_gen_meshes(C.byref(p), w, None, 0, None, None, 0, None, C.byref(nv), C.byref(nf), C.byref(no), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode())
    V = np.empty((nv.value, 3), np.float32)
    F = np.empty((nf.value, 3), np.uint32)
    vo = np.empty(no.value + 1, np.int64)
    fo = np.empty(no.value + 1, np.int64)
    rc = L.tdp_gen_meshes(C.byref(p), w, _ptr(V), V.size, _ptr(vo), _ptr(F), F.size, _ptr(fo), C.byref(nv),
                          C.byref(nf), C.byref(no), err, 512)
    if rc != TDP_OK:
        raise TdpError(rc, err.value.decode())
    return V, vo, F, fo


def read_off(path_or_text):
    """One OFF polyhedron (the reference's mesh text format, as in its data/*.pt
    prototypes) -> (vertices[n, 3] float32, triangles[m, 3] uint32).  Polygons
    with more than three corners are fanned from their first corner."""
    text = path_or_text
    if isinstance(path_or_text, (str, os.PathLike)) and Path(path_or_text).exists():
        text = Path(path_or_text).read_text()
    tok = []
    for line in str(text).splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            tok.extend(line.split())
    if not tok or tok[0] != "OFF":
        raise ValueError("not an OFF mesh")
    nv, nf = int(tok[1]), int(tok[2])
    at = 4
    V = np.array(tok[at:at + 3 * nv], np.float32).reshape(nv, 3)
    at += 3 * nv
    tris = []
    for _ in range(nf):
        k = int(tok[at])
        idx = [int(x) for x in tok[at + 1:at + 1 + k]]
        at += 1 + k
        for j in range(1, k - 1):
            tris.append((idx[0], idx[j], idx[j + 1]))
    return V, np.array(tris, np.uint32).reshape(-1, 3)


def stack_meshes(meshes):
    """[(vertices, triangles), ...] -> (vertices, vert_off, faces, face_off) for raw_from_meshes."""
    vs = [np.asarray(v, np.float32).reshape(-1, 3) for v, _ in meshes]
    fs = [np.asarray(f, np.uint32).reshape(-1, 3) for _, f in meshes]
    vo = np.concatenate([[0], np.cumsum([len(v) for v in vs])]).astype(np.int64)
    fo = np.concatenate([[0], np.cumsum([len(f) for f in fs])]).astype(np.int64)
    V = np.concatenate(vs) if vs else np.zeros((0, 3), np.float32)
    F = np.concatenate(fs) if fs else np.zeros((0, 3), np.uint32)
    return V, vo, F, fo
