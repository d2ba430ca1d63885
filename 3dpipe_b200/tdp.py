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
QUERY_NN, QUERY_WITHIN = 1, 2

# Every symbol include/tdp.h declares; tests check the library exports them all.
EXPORTED = [
    "tdp_ctx_create", "tdp_ctx_destroy", "tdp_last_error", "tdp_ctx_memory", "tdp_last_stats",
    "tdp_refine_batch",
]


class TdpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [("refine_ms", C.c_double), ("filter_ms", C.c_double), ("total_ms", C.c_double),
                ("full_evals", C.c_ulonglong), ("tri_pairs", C.c_double), ("refine_items", C.c_long),
                ("refine_launches", C.c_long), ("recheck_pairs", C.c_long), ("filter_pairs", C.c_long),
                ("filter_voxel_pairs", C.c_double), ("kernel_launches", C.c_long)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


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
    _lib = L
    return L


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """A device context: stream, memory budget, scratch buffers."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        L = lib()
        h = C.c_void_p()
        rc = L.tdp_ctx_create(device, budget_bytes, 0, C.byref(h))
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
