"""GPU LOD preparation (tdp_raw_from_meshes): LOD-100 meshes in, a RAW tile out.

CPU tests pin the oracle (oracle/lodprep_oracle.cpp, a priority-queue
decimation) against an independent Python restatement that runs the rule the
way the GPU does (tests/lodprep_py.py, refused-edge flags and a full argmin per
round), byte for byte, and check the oracle's tiles: they parse, their LODs
shrink to the targets, every LOD of a closed mesh stays closed, and the bounds
computed on them are conservative.  GPU tests require the device output to
equal the oracle's tile with the bound oracle applied, byte for byte, for the
generator's nuclei and vessels and for edge cases (a tetrahedron that cannot
shrink, an open patch, a flat disc, separate components, an object of more
than 65,535 vertices, objects split over several batches), report bad objects
like the oracle, and give tiles whose join equals the reference rules.
"""
import ctypes as C

import numpy as np
import pytest

import lodprep_py
from oracle_bind import oracle
from rawdt import read_tile

P = C.c_void_p


# ------------------------------------------------------------------ meshes
def icosphere(subdiv, radius=10.0, centre=(0.0, 0.0, 0.0), jitter=0.0, seed=0):
    t = (1 + 5 ** 0.5) / 2
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    V = [np.array(v, float) / np.linalg.norm(v) for v in V]
    for _ in range(subdiv):
        mid, G = {}, []

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = V[a] + V[b]
                V.append(p / np.linalg.norm(p))
                mid[k] = len(V) - 1
            return mid[k]

        for a, b, c in F:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            G += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = G
    V = np.array(V) * radius
    if jitter:
        V *= 1 + jitter * np.random.default_rng(seed).uniform(-1, 1, (len(V), 1))
    return (V + np.array(centre)).astype(np.float32), np.array(F, np.uint32)


def grid_patch(k, flat=False, seed=0):
    """open (k+1) x (k+1) vertex patch, 2 k^2 triangles"""
    g = np.random.default_rng(seed)
    xs, ys = np.meshgrid(np.arange(k + 1, dtype=float), np.arange(k + 1, dtype=float), indexing="ij")
    z = np.zeros_like(xs) if flat else 0.3 * np.sin(xs / 2) * np.cos(ys / 3) + 0.01 * g.standard_normal(xs.shape)
    V = np.stack([xs, ys, z], -1).reshape(-1, 3).astype(np.float32)
    F = []
    for i in range(k):
        for j in range(k):
            a, b, c, d = i * (k + 1) + j, (i + 1) * (k + 1) + j, (i + 1) * (k + 1) + j + 1, i * (k + 1) + j + 1
            F += [(a, b, c), (a, c, d)]
    return V, np.array(F, np.uint32)


def tetrahedron():
    V = np.array([(0, 0, 0), (4, 0, 0), (0, 4, 0), (0, 0, 4)], np.float32)
    F = np.array([(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)], np.uint32)
    return V, F


def two_spheres():
    V1, F1 = icosphere(1, 5, (0, 0, 0), 0.05, 1)
    V2, F2 = icosphere(1, 5, (30, 0, 0), 0.05, 2)
    return np.concatenate([V1, V2]), np.concatenate([F1, F2 + len(V1)])


def spare_vertices(n_total=70000):
    """a small sphere whose vertex array also holds unreferenced vertices, so
    the object has more than 65,535 vertices (32-bit ids, global storage)"""
    V, F = icosphere(2, 8, (100, 50, 0), 0.1, 3)
    g = np.random.default_rng(4)
    extra = (g.uniform(-1, 1, (n_total - len(V), 3)) * 3 + np.array([100, 50, 0])).astype(np.float32)
    return np.concatenate([V, extra]), F


def small_cases():
    return [icosphere(2, 10, (0, 0, 0), 0.08, 7), icosphere(1, 6, (40, 0, 0), 0.2, 8), tetrahedron(),
            grid_patch(6, seed=9), grid_patch(5, flat=True), two_spheres()]


# ------------------------------------------------------------------ oracle
def stack(meshes):
    vs = [np.asarray(v, np.float32).reshape(-1, 3) for v, _ in meshes]
    fs = [np.asarray(f, np.uint32).reshape(-1, 3) for _, f in meshes]
    vo = np.concatenate([[0], np.cumsum([len(v) for v in vs])]).astype(np.int64)
    fo = np.concatenate([[0], np.cumsum([len(f) for f in fs])]).astype(np.int64)
    return np.ascontiguousarray(np.concatenate(vs)), vo, np.ascontiguousarray(np.concatenate(fs)), fo


def oracle_prep(meshes, voxel_size=100, threads=0):
    """the oracle's tile (zero bounds), or the oracle's return code"""
    V, vo, F, fo = stack(meshes)
    L = oracle().L
    L.tdo_raw_from_meshes.argtypes = [P, P, P, P, C.c_long, C.c_int, P, C.c_size_t, C.POINTER(C.c_size_t), C.c_int]
    L.tdo_raw_from_meshes.restype = C.c_long
    n = C.c_size_t()
    rc = L.tdo_raw_from_meshes(V.ctypes.data, vo.ctypes.data, F.ctypes.data, fo.ctypes.data, len(vo) - 1,
                               voxel_size, None, 0, C.byref(n), threads)
    if rc != 0:
        return rc
    out = np.empty(n.value, np.uint8)
    rc = L.tdo_raw_from_meshes(V.ctypes.data, vo.ctypes.data, F.ctypes.data, fo.ctypes.data, len(vo) - 1,
                               voxel_size, out.ctypes.data, out.size, C.byref(n), threads)
    assert rc == 0
    return out


def with_bounds(raw):
    from test_bounds import oracle_bounds
    return oracle_bounds(raw)


def _lod_counts(raw):
    return [[sum(len(t) for t in o.tris[li]) for li in range(5)] for o in read_tile(raw)]


# ------------------------------------------------------------------ CPU: the oracle
@pytest.mark.parametrize("case", range(6))
def test_oracle_equals_independent_restatement(case):
    mesh = small_cases()[case]
    for vs in (100, 40):
        want = lodprep_py.prepare([mesh], vs)
        got = oracle_prep([mesh], vs)
        assert bytes(got) == want, (case, vs)


def test_oracle_tile_parses_and_shrinks(pkg):
    meshes = small_cases()
    raw = oracle_prep(meshes, 40)
    assert pkg.tdp.raw_check(raw)[0] == len(meshes)
    for (V, F), cnt in zip(meshes, _lod_counts(raw)):
        assert cnt[4] == len(F)
        assert all(cnt[i] <= cnt[i + 1] for i in range(4))
    # the sphere reaches every target; the tetrahedron cannot shrink at all
    assert _lod_counts(raw)[0][:4] == [64, 128, 192, 256]
    assert _lod_counts(raw)[2] == [4, 4, 4, 4, 4]


def test_oracle_lods_of_closed_meshes_stay_closed():
    from collections import Counter
    V, F = icosphere(2, 10, (0, 0, 0), 0.08, 7)
    o = read_tile(oracle_prep([(V, F)], 100))[0]
    for li in range(4):
        tris = np.concatenate(o.tris[li]).reshape(-1, 3, 3)
        edges = Counter()
        for t in tris:
            for j in range(3):
                a, b = tuple(t[j]), tuple(t[(j + 1) % 3])
                edges[(min(a, b), max(a, b))] += 1
        assert set(edges.values()) == {2}, li   # every edge has two facets


def test_oracle_bounds_are_conservative_on_prepared_tiles():
    from test_bounds import violation
    raw = with_bounds(oracle_prep(small_cases()[:2] + [two_spheres()], 40))
    # FP64 rounding of the sampled distances only (coordinates up to ~1e2)
    assert violation(raw, samples=4).max() <= 1e-9


def test_oracle_reports_the_first_bad_object():
    good = icosphere(1)
    bad_index = (good[0], np.array([[0, 1, 99]], np.uint32))
    repeat = (good[0], np.array([[0, 1, 1]], np.uint32))
    empty = (good[0], np.zeros((0, 3), np.uint32))
    assert oracle_prep([good, good, bad_index, repeat]) == -3
    assert oracle_prep([good, repeat]) == -2
    assert oracle_prep([empty]) == -1


def test_prep_bound_and_generator_meshes(pkg):
    """raw_prep_bound holds the tile; the generator's meshes are the objects of
    its tiles (same float vertices, LOD-100 facet for facet)"""
    V, vo, F, fo = pkg.tdp.gen_meshes(2, 3, seed=11, which="nuclei")
    assert len(vo) == 7 and (np.diff(fo) == 1280).all()
    meshes = [(V[vo[i]:vo[i + 1]], F[fo[i]:fo[i + 1]]) for i in range(len(vo) - 1)]
    raw = oracle_prep(meshes[:2], 100)
    assert raw.size <= pkg.tdp.raw_prep_bound(fo[:3], 100)
    nb, _ = pkg.tdp.gen_tiles(2, 3, seed=11)
    objs = read_tile(nb)
    for i, o in enumerate(objs):
        got = np.sort(np.concatenate(o.tris[4]).reshape(-1, 9), axis=0)
        Vi, Fi = meshes[i]
        want = np.sort(Vi[Fi].reshape(-1, 9), axis=0)
        np.testing.assert_array_equal(got, want)
    Vv, vov, Fv, fov = pkg.tdp.gen_meshes(2, 3, seed=11, which="vessels")
    assert len(vov) == 3 and fov[1] > 10000
    with pytest.raises(pkg.TdpError):
        pkg.tdp.raw_prep_bound(np.array([0, 5, 3]), 100)


# ------------------------------------------------------------------ GPU
def _gpu(ctx, meshes, vs=100):
    import importlib
    tdp = importlib.import_module("3dpipe_b200").tdp
    raw, info = ctx.raw_from_meshes(*tdp.stack_meshes(meshes), voxel_size=vs)
    return np.array(raw), info


@pytest.mark.gpu
def test_gpu_prep_equals_oracle_on_generated_objects(pkg, ctx):
    V, vo, F, fo = pkg.tdp.gen_meshes(3, 4, seed=21, which="nuclei")
    nuclei = [(V[vo[i]:vo[i + 1]], F[fo[i]:fo[i + 1]]) for i in range(len(vo) - 1)]
    Vv, vov, Fv, fov = pkg.tdp.gen_meshes(3, 4, seed=21, which="vessels")
    vessels = [(Vv[vov[i]:vov[i + 1]], Fv[fov[i]:fov[i + 1]]) for i in range(len(vov) - 1)]
    for meshes in (nuclei, vessels[:2]):
        got, info = _gpu(ctx, meshes)
        want = with_bounds(oracle_prep(meshes))
        assert got.size == want.size and np.array_equal(got, want)
        assert info["n_objects"] == len(meshes) and info["n_triangles"][4] == sum(len(f) for _, f in meshes)


@pytest.mark.gpu
@pytest.mark.parametrize("vs", [100, 40, 7])
def test_gpu_prep_equals_oracle_on_edge_cases(ctx, vs):
    meshes = small_cases()
    got, _ = _gpu(ctx, meshes, vs)
    assert np.array_equal(got, with_bounds(oracle_prep(meshes, vs)))


@pytest.mark.gpu
def test_gpu_prep_wide_object_ids(ctx):
    meshes = [spare_vertices(), icosphere(2, 10, (0, 0, 0), 0.08, 7)]
    got, _ = _gpu(ctx, meshes)
    assert np.array_equal(got, with_bounds(oracle_prep(meshes)))


@pytest.mark.gpu
def test_gpu_prep_batches_equal_one_batch(pkg):
    """a context with a small memory cap splits the objects into batches; the
    tile is the same"""
    V, vo, F, fo = pkg.tdp.gen_meshes(15, 10, seed=31, which="nuclei")
    small = pkg.Context(0, budget_bytes=256 << 20)
    try:
        raw_b, info_b = small.raw_from_meshes(V, vo, F, fo)
    finally:
        small.close()
    assert info_b["batches"] >= 2
    meshes = [(V[vo[i]:vo[i + 1]], F[fo[i]:fo[i + 1]]) for i in range(len(vo) - 1)]
    assert np.array_equal(np.array(raw_b), with_bounds(oracle_prep(meshes)))


@pytest.mark.gpu
def test_gpu_prep_reports_bad_objects(pkg, ctx):
    good = icosphere(1)
    for meshes, first in (([good, (good[0], np.array([[0, 1, 99]], np.uint32))], 1),
                          ([good, good, (good[0], np.array([[0, 2, 2]], np.uint32))], 2),
                          ([(good[0] * np.float32(np.nan), good[1])], 0)):
        with pytest.raises(pkg.TdpError) as e:
            _gpu(ctx, meshes)
        assert e.value.code == 1 and ("object %d " % first) in str(e.value)
    # the context stays usable
    got, _ = _gpu(ctx, [good])
    assert np.array_equal(got, with_bounds(oracle_prep([good])))


@pytest.mark.gpu
def test_join_on_prepared_tiles_equals_reference_rules(pkg, ctx):
    from oracle_bind import ref_join
    V, vo, F, fo = pkg.tdp.gen_meshes(2, 6, seed=41, which="nuclei")
    Vv, vov, Fv, fov = pkg.tdp.gen_meshes(2, 6, seed=41, which="vessels", tube_sides=10, tube_rings=16)
    nb, _ = ctx.raw_from_meshes(V, vo, F, fo)
    vb, _ = ctx.raw_from_meshes(Vv, vov, Fv, fov)
    nb, vb = np.array(nb), np.array(vb)
    T1, T2 = pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb)
    try:
        for kw in (dict(query="nn", knn=2), dict(query="within", within=120.0)):
            q, t, _ = ctx.join(T1, T2, form=pkg.FORM_TUNED, **kw)
            r = ref_join(nb, vb, False, kw["query"] == "nn", knn=kw.get("knn", 0), tau=kw.get("within", 0.0))
            if r is not None:
                assert set(zip(q.tolist(), t.tolist())) == set(zip(r[0].tolist(), r[1].tolist()))
            assert len(q) > 0
    finally:
        T1.free()
        T2.free()
