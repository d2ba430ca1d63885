"""ctypes bindings of the test-only checkers: the FP64 oracle (oracle/liboracle.so)
and the reference's own CPU code compiled from source (oracle/_ref/libtdp_ref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libtdp_ref.so"
P = C.c_void_p


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        L = C.CDLL(str(path))
        L.tdo_tri_dist.argtypes = [P, P]
        L.tdo_tri_dist.restype = C.c_double
        L.tdo_tri_dist_batch.argtypes = [P, P, C.c_size_t, P, P]
        L.tdo_voxel_pair.argtypes = [P, P, C.c_size_t, P, P, C.c_size_t, P]
        self.L = L

    def tri_dist_batch(self, S, T):
        S = np.ascontiguousarray(S, np.float64).reshape(-1, 9)
        T = np.ascontiguousarray(T, np.float64).reshape(-1, 9)
        a = np.empty(len(S))
        b = np.empty(len(S))
        self.L.tdo_tri_dist_batch(_p(S), _p(T), len(S), _p(a), _p(b))
        return a, b

    def voxel_pair(self, t1, h1, t2, h2):
        t1 = np.ascontiguousarray(t1, np.float32).reshape(-1, 9)
        t2 = np.ascontiguousarray(t2, np.float32).reshape(-1, 9)
        h1 = None if h1 is None else np.ascontiguousarray(h1, np.float32).reshape(-1, 2)
        h2 = None if h2 is None else np.ascontiguousarray(h2, np.float32).reshape(-1, 2)
        out = np.empty(3)
        self.L.tdo_voxel_pair(_p(t1), None if h1 is None else _p(h1), len(t1),
                              _p(t2), None if h2 is None else _p(h2), len(t2), _p(out))
        return out


class Reference:
    def __init__(self, path=REF_SO):
        L = C.CDLL(str(path))
        L.tdr_tri_dist_batch.argtypes = [P, P, C.c_size_t, P]
        L.tdr_mesh_dist.argtypes = [P, P, C.c_size_t, C.c_size_t, P, P, P]
        L.tdr_candidates.argtypes = [P, P, C.c_long, P, P, C.c_long, C.c_int, C.c_int, C.c_float, C.c_int,
                                     P, P, C.c_long]
        L.tdr_candidates.restype = C.c_long
        self.L = L

    def tri_dist_batch(self, S, T):
        S = np.ascontiguousarray(S, np.float32).reshape(-1, 9)
        T = np.ascontiguousarray(T, np.float32).reshape(-1, 9)
        out = np.empty(len(S), np.float32)
        self.L.tdr_tri_dist_batch(_p(S), _p(T), len(S), _p(out))
        return out

    def mesh_dist(self, t1, t2, h1, h2):
        t1 = np.ascontiguousarray(t1, np.float32)
        t2 = np.ascontiguousarray(t2, np.float32)
        h1 = np.ascontiguousarray(h1, np.float32)
        h2 = np.ascontiguousarray(h2, np.float32)
        out = np.empty(3, np.float32)
        self.L.tdr_mesh_dist(_p(t1), _p(t2), len(t1), len(t2), _p(h1), _p(h2), _p(out))
        return out

    def candidates(self, box1, xf1, box2, xf2, self_join, knn, within, is_knn):
        box1 = np.ascontiguousarray(box1, np.float32)
        xf1 = np.ascontiguousarray(xf1, np.float32)
        box2 = np.ascontiguousarray(box2, np.float32)
        xf2 = np.ascontiguousarray(xf2, np.float32)
        n1, n2 = len(box1), len(box2)
        cap = max(1024, n1 * 64)
        while True:
            off = np.zeros(n1 + 1, np.int64)
            ids = np.zeros(cap, np.int32)
            tot = self.L.tdr_candidates(_p(box1), _p(xf1), n1, _p(box2), _p(xf2), n2, int(self_join), int(knn),
                                        float(within), int(is_knn), _p(off), _p(ids), cap)
            if tot >= 0:
                return off, ids[:tot].copy()
            cap *= 4


def oracle():
    if not ORACLE_SO.exists():
        raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
    return Oracle()


def reference():
    return Reference() if REF_SO.exists() else None


def join_exact(tile1, tile2, self_join, is_knn, knn=1, tau=0.0, threads=0):
    """FP64 exact join: every evaluated (q, t, D, in_result) as numpy arrays."""
    O = oracle()
    L = O.L
    L.tdo_join_exact.argtypes = [P, C.c_size_t, P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                 P, P, P, P, C.c_long]
    L.tdo_join_exact.restype = C.c_long
    t1 = np.ascontiguousarray(tile1, np.uint8)
    t2 = t1 if tile2 is None else np.ascontiguousarray(tile2, np.uint8)
    cap = 1 << 16
    while True:
        q = np.empty(cap, np.int32); t = np.empty(cap, np.int32); d = np.empty(cap); i = np.empty(cap, np.int32)
        n = L.tdo_join_exact(_p(t1), t1.size, _p(t2), t2.size, int(self_join), int(is_knn), int(knn), float(tau),
                             int(threads), _p(q), _p(t), _p(d), _p(i), cap)
        if n >= 0:
            return q[:n], t[:n], d[:n], i[:n].astype(bool)
        cap = -n


def ref_join(tile1, tile2, self_join, is_knn, knn=1, tau=0.0, lods=None, level=2, threads=0, max_queries=0,
             queries=None):
    """The reference's join rules on the CPU with the reference's own MeshDist/octree.
    max_queries > 0 joins only the first max_queries query objects; `queries`
    (ids into tile 1) joins only those (each query's candidate list and result
    are the ones the whole join gives it).
    Returns (q, t, stats) with stats = (seconds, tri_pairs, voxel_pairs_refined, candidates)."""
    R = reference()
    if R is None:
        return None
    L = R.L
    L.tdr_join.argtypes = [P, C.c_size_t, P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_float, P, C.c_int, C.c_int,
                           C.c_int, C.c_long, P, P, C.c_long, P]
    L.tdr_join.restype = C.c_long
    L.tdr_join_sel.argtypes = [P, C.c_size_t, P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_float, P, C.c_int,
                               C.c_int, C.c_int, P, C.c_long, P, P, C.c_long, P]
    L.tdr_join_sel.restype = C.c_long
    t1 = np.ascontiguousarray(tile1, np.uint8)
    t2 = t1 if tile2 is None else np.ascontiguousarray(tile2, np.uint8)
    lods = np.array(lods or [20, 40, 60, 80, 100], np.int32)
    qsel = None if queries is None else np.ascontiguousarray(queries, np.int32)
    if qsel is not None and len(qsel) == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(4)
    cap = 1 << 16
    while True:
        q = np.empty(cap, np.int32); t = np.empty(cap, np.int32); st = np.zeros(4)
        if qsel is None:
            n = L.tdr_join(_p(t1), t1.size, _p(t2), t2.size, int(self_join), int(is_knn), int(knn), float(tau),
                           _p(lods), len(lods), int(level), int(threads), int(max_queries), _p(q), _p(t), cap, _p(st))
        else:
            n = L.tdr_join_sel(_p(t1), t1.size, _p(t2), t2.size, int(self_join), int(is_knn), int(knn), float(tau),
                               _p(lods), len(lods), int(level), int(threads), _p(qsel), len(qsel), _p(q), _p(t), cap,
                               _p(st))
        if n >= 0:
            o = np.lexsort((t[:n], q[:n]))
            return q[:n][o], t[:n][o], st
        cap = -n


def ref_join_capped(tile1, tile2, self_join, tau, cap_rel, lods=None, threads=0):
    """The within join of the reference rules (level 2) with a cap replayed on
    the LODs before the last (ref_join.cpp, join_impl): a voxel pair whose
    Hausdorff lower bound comes out above the pair's cap keeps its previous
    bounds.  Returns (q, t, (capped voxel-pair refines, their triangle pairs))."""
    R = reference()
    if R is None:
        return None
    L = R.L
    L.tdr_join_capped.argtypes = [P, C.c_size_t, P, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_float, P, C.c_int,
                                  C.c_int, C.c_int, C.c_float, P, P, C.c_long, P, P]
    L.tdr_join_capped.restype = C.c_long
    t1 = np.ascontiguousarray(tile1, np.uint8)
    t2 = t1 if tile2 is None else np.ascontiguousarray(tile2, np.uint8)
    lods = np.array(lods or [20, 40, 60, 80, 100], np.int32)
    cap = 1 << 16
    while True:
        q = np.empty(cap, np.int32); t = np.empty(cap, np.int32); st = np.zeros(4); cs = np.zeros(2)
        n = L.tdr_join_capped(_p(t1), t1.size, _p(t2), t2.size, int(self_join), 0, 0, float(tau), _p(lods),
                              len(lods), 2, int(threads), float(cap_rel), _p(q), _p(t), cap, _p(st), _p(cs))
        if n >= 0:
            o = np.lexsort((t[:n], q[:n]))
            return q[:n][o], t[:n][o], cs
        cap = -n

