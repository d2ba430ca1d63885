"""Bound preparation: the per-triangle (proxy, hausdorff) bounds computed on the
GPU (tdp_tile_compute_bounds / tdp_raw_compute_bounds) against the FP64 CPU
restatement in oracle/bounds_oracle.cpp.

CPU tests pin the oracle itself: its pruned search equals a brute-force scan,
and the bounds it produces are conservative (sampled points, and the object-pair
rule d_LOD - ph1 - ph2 <= d_100 <= d_LOD + h1 + h2 that the join relies on).
GPU tests require the device bounds to equal the oracle's bit for bit (RAW
bytes compared whole), including hand-made edge cases, and a join on tiles
whose bounds came from the GPU to return the FP64 exact result set.
"""
import ctypes as C
import numpy as np
import pytest

from join_cases import exact_truth
from oracle_bind import oracle
from rawdt import read_tile, write_tile as make_raw

P = C.c_void_p


def _lib():
    L = oracle().L
    L.tdo_tile_bounds.argtypes = [P, C.c_size_t, P, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.tdo_bounds_violation.argtypes = [P, C.c_size_t, C.c_int, C.c_uint64, P]
    return L


def oracle_bounds(raw, prune=True, threads=0):
    raw = np.ascontiguousarray(raw, np.uint8)
    out = np.empty_like(raw)
    ev = C.c_double()
    assert _lib().tdo_tile_bounds(raw.ctypes.data, raw.size, out.ctypes.data, int(prune), threads, C.byref(ev)) == 0
    return out


def violation(raw, samples=3, seed=5):
    raw = np.ascontiguousarray(raw, np.uint8)
    v = np.zeros(2)
    assert _lib().tdo_bounds_violation(raw.ctypes.data, raw.size, samples, seed, v.ctypes.data) == 0
    return v


def small_tiles(pkg, seed=11):
    return pkg.tdp.gen_tiles(1, 4, seed=seed, tube_sides=8, tube_rings=12)


def edge_case_tile(pkg):
    """Hand-made objects: an object with no LOD-20 triangle, a voxel empty at
    some LODs, zero-area triangles at LOD 40 and LOD 100, and an object whose
    LOD 100 is empty (no surface: its bounds are 0)."""
    nb, _ = pkg.tdp.gen_tiles(1, 2, seed=3)
    N = read_tile(nb)
    a = N[0]
    objs = []
    # object 0: generated nucleus, LOD 20 emptied
    objs.append([[np.zeros((0, 9), np.float32) for _ in a.tris[0]]] + [list(a.tris[li]) for li in range(1, 5)])
    # object 1: second nucleus with voxel 0 emptied at LODs 20 and 60, plus degenerate triangles
    b = N[1]
    o1 = [list(b.tris[li]) for li in range(5)]
    o1[0][0] = np.zeros((0, 9), np.float32)
    o1[2][0] = np.zeros((0, 9), np.float32)
    t40 = o1[1][1].copy()
    t40[0, 6:9] = t40[0, 0:3]                                   # two equal vertices
    t40[1, 3:6] = (t40[1, 0:3] + t40[1, 6:9]) / 2               # collinear vertices
    o1[1][1] = t40
    t100 = o1[4][2].copy()
    t100[0, 3:9] = np.tile(t100[0, 0:3], 2)                     # a point
    o1[4][2] = t100
    objs.append(o1)
    # object 2: a single voxel with LOD 20-80 triangles and no LOD-100 facet
    tri = np.array([[0, 0, 0, 10, 0, 0, 0, 10, 0], [0, 0, 5, 10, 0, 5, 0, 10, 5]], np.float32)
    objs.append([[tri], [tri], [tri[:1]], [tri], [np.zeros((0, 9), np.float32)]])
    return make_raw(objs)


# ------------------------------------------------------------------ CPU: the oracle


def test_bounds_oracle_pruned_equals_brute_force(pkg):
    nb, vb = small_tiles(pkg)
    for raw in (nb, vb, edge_case_tile(pkg)):
        np.testing.assert_array_equal(oracle_bounds(raw, prune=True), oracle_bounds(raw, prune=False))


def test_bounds_oracle_are_conservative(pkg):
    nb, vb = small_tiles(pkg)
    for raw in (nb, vb):
        b = oracle_bounds(raw)
        v = violation(b)
        # FP64 rounding of the sampled distances only (coordinates up to ~1e3)
        assert v[0] <= 1e-9 and v[1] <= 1e-9, v
        # the object-pair rule the join relies on (LOD-100 distance in FP64)
        O = oracle()
        N = read_tile(b)
        for i, j in [(0, 1), (2, 3), (0, 3)]:
            if j >= len(N):
                continue
            x, y = N[i], N[j]
            d100 = O.voxel_pair(x.lod_tris(4), None, y.lod_tris(4), None)[0]
            for li in range(4):
                r = O.voxel_pair(x.lod_tris(li), np.concatenate(x.hds[li]), y.lod_tris(li), np.concatenate(y.hds[li]))
                assert r[1] <= d100 + 1e-9 <= r[2] + 2e-9, (i, j, li, r, d100)


def test_bounds_oracle_object_level_and_edge_cases(pkg):
    raw = edge_case_tile(pkg)
    N = read_tile(oracle_bounds(raw))
    for o in N:
        for li in range(5):
            h = np.concatenate(o.hds[li]) if o.tris[li] else np.zeros((0, 2), np.float32)
            assert o.hausdorff[li] == (h[:, 1].max() if len(h) else 0.0)
            assert o.proxyhausdorff[li] == (h[:, 0].max() if len(h) else 0.0)
        assert all(not len(h) or not h.any() for h in o.hds[4])   # LOD 100: 0
    assert N[0].hausdorff[0] == 0 and N[0].proxyhausdorff[0] == 0  # no LOD-20 triangle
    assert not np.concatenate(N[2].hds[0]).any()                   # no surface, no bound
    assert np.isfinite(np.concatenate(N[1].hds[1])).all()          # degenerate triangles measured


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
def test_gpu_bounds_equal_oracle_bit_for_bit(pkg, ctx):
    nb, vb = small_tiles(pkg)
    nb2, vb2 = pkg.tdp.gen_tiles(1, 6, seed=29)
    for raw in (nb, vb, nb2, vb2, edge_case_tile(pkg)):
        got, info = ctx.raw_compute_bounds(raw)
        want = oracle_bounds(raw)
        assert np.array_equal(got, want), "GPU bounds differ from the oracle"
        assert info["objects"] == len(read_tile(raw)) and info["dist_evals"] > 0
        # in place, and idempotent
        again = got.copy()
        ctx.raw_compute_bounds(again, out=again)
        np.testing.assert_array_equal(again, got)


@pytest.mark.gpu
def test_tile_bounds_in_place_equal_raw_path(pkg, ctx):
    nb, vb = pkg.tdp.gen_tiles(2, 10, seed=41)
    T1, T2 = pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb)
    info = ctx.compute_bounds(T1)
    ctx.compute_bounds(T2)
    assert info["triangles"] == sum(T1.info()["n_tris"][:4]) and info["facet_queries"] > 0 and info["pieces"] > 0
    r1, _ = ctx.raw_compute_bounds(nb)
    r2, _ = ctx.raw_compute_bounds(vb)
    U1, U2 = pkg.tdp.Tile(ctx, r1), pkg.tdp.Tile(ctx, r2)
    for args in (dict(query="nn", knn=3), dict(query="within", within=150.0)):
        a = ctx.join(T1, T2, **args)
        b = ctx.join(U1, U2, **args)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("query,knn,tau", [("nn", 2, 0.0), ("nn", 4, 0.0), ("within", 1, 150.0), ("within", 1, 400.0)])
def test_join_on_gpu_bounds_returns_exact_set(pkg, ctx, query, knn, tau):
    nb, vb = pkg.tdp.gen_tiles(6, 8, seed=57)
    rn, _ = ctx.raw_compute_bounds(nb)
    rv, _ = ctx.raw_compute_bounds(vb)
    truth, margin = exact_truth(nb, vb, False, query, knn, tau)
    assert margin > 1e-3
    T1, T2 = pkg.tdp.Tile(ctx, rn), pkg.tdp.Tile(ctx, rv)
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        q, t, _ = ctx.join(T1, T2, query=query, knn=knn, within=tau, form=form)
        assert set(zip(q.tolist(), t.tolist())) == truth, form
