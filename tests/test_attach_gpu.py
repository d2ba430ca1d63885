"""Attached tiles (tdp_tile_attach): the triangles stay in page-locked host
memory and each join fetches the voxels its refine touches.  Every join on
attached tiles must return exactly what the same join on uploaded tiles
returns (ids, distances, exact FP64 distances), fetch only part of the tile,
and fetch nothing the second time; attach refuses unlocked memory and tiles
not in the writer's layout.  The context poisons attached records with NaN,
so a record that no fetch filled would change the results."""
import numpy as np
import pytest

from join_cases import CASES, tiles
from rawdt import read_tile, write_tile

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pctx(pkg):
    c = pkg.Context(0, 0, pkg.tdp.CTX_POISON)
    yield c
    c.close()


def both(pkg, ctx, nb, vb):
    up = (pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb))
    pn, pv = pkg.tdp.pinned_copy(nb), pkg.tdp.pinned_copy(vb)
    at = (pkg.tdp.Tile(ctx, pn, attach=True), pkg.tdp.Tile(ctx, pv, attach=True))
    return up, at


def same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", list(CASES))
def test_attached_join_equals_uploaded(pkg, pctx, name):
    nv, npv, seed, query, knn, tau, self_join, lods, level = CASES[name]
    nb, vb = tiles(nv, npv, seed)
    U1, U2 = pkg.tdp.Tile(pctx, nb), pkg.tdp.Tile(pctx, vb)
    pn, pv = pkg.tdp.pinned_copy(nb), pkg.tdp.pinned_copy(vb)
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        args = dict(query=query, knn=knn, within=tau, lods=lods, hausdorff_level=level, form=form)
        want = pctx.join(U1, None if self_join else U2, **args)
        assert pctx.stats()["fetch_bytes"] == 0
        # freshly attached tiles per form: nothing fetched yet
        A1, A2 = pkg.tdp.Tile(pctx, pn, attach=True), pkg.tdp.Tile(pctx, pv, attach=True)
        got = pctx.join(A1, None if self_join else A2, **args)
        st = pctx.stats()
        assert st["refine_items"] == 0 or st["fetch_bytes"] > 0
        same(got, want)
        A1.free()
        A2.free()
    U1.free()
    U2.free()


def test_attached_fetches_part_once(pkg, pctx):
    nb, vb = tiles(6, 12, 101)
    (U1, U2), (A1, A2) = both(pkg, pctx, nb, vb)
    info = A1.info()
    assert info["attached"] and not U1.info()["attached"]
    assert info["h2d_bytes"] < nb.size // 10
    args = dict(query="within", within=400.0, exact_distances=True)
    want = pctx.join(U1, U2, **args)
    got = pctx.join(A1, A2, **args)
    same(got, want)
    st = pctx.stats()
    assert 0 < st["fetch_bytes"] < (nb.size + vb.size) / 2, st["fetch_bytes"]
    again = pctx.join(A1, A2, **args)
    same(again, want)
    assert pctx.stats()["fetch_bytes"] == 0          # every voxel it needs is resident now
    # other queries on the same attached tiles still agree
    same(pctx.join(A1, A2, query="within", within=150.0), pctx.join(U1, U2, query="within", within=150.0))
    same(pctx.join(A1, A2, query="nn", knn=5), pctx.join(U1, U2, query="nn", knn=5))
    for T in (U1, U2, A1, A2):
        T.free()


def test_attached_exact_mixed_and_graph(pkg, pctx):
    nb, vb = tiles(6, 12, 101)
    (U1, U2), (A1, A2) = both(pkg, pctx, nb, vb)
    want = pctx.join(U1, U2, query="within", within=400.0, exact_distances=True)
    got = pctx.join(A1, A2, query="within", within=400.0, exact_distances=True)
    same(got, want)
    n1 = U1.info()["n_objects"]
    rng = np.random.default_rng(3)
    ok = rng.integers(0, 4, n1).astype(np.int32)
    ow = np.where(ok == 0, 120.0, 0.0).astype(np.float32)
    same(pctx.join(A1, A2, obj_knn=ok, obj_within=ow), pctx.join(U1, U2, obj_knn=ok, obj_within=ow))
    # repeated joins replay the LOD graph with the fetch step inside it
    pctx.set_lod_graph(pkg.tdp.LOD_GRAPH_ALWAYS)
    try:
        for _ in range(2):
            same(pctx.join(A1, A2, query="nn", knn=2), pctx.join(U1, U2, query="nn", knn=2))
    finally:
        pctx.set_lod_graph(pkg.tdp.LOD_GRAPH_AUTO)
    for T in (U1, U2, A1, A2):
        T.free()


def test_attached_bounds_equal_uploaded(pkg, pctx):
    nb, vb = pkg.tdp.gen_tiles(1, 5, seed=13)
    U = pkg.tdp.Tile(pctx, nb)
    A = pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(nb), attach=True)
    pctx.compute_bounds(U)
    pctx.compute_bounds(A)
    V = pkg.tdp.Tile(pctx, vb)
    same(pctx.join(A, V, query="nn", knn=1), pctx.join(U, V, query="nn", knn=1))
    for T in (U, A, V):
        T.free()


def test_attach_refusals(pkg, pctx):
    nb, _ = tiles(2, 4, 7)
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.Tile(pctx, np.array(nb), attach=True)          # pageable memory
    assert e.value.code == 1
    N = read_tile(nb)
    objs = [[list(o.tris[li]) for li in range(5)] for o in N[:2]]
    shuffled = write_tile(objs, lod_order=(4, 3, 2, 1, 0))     # valid RAW, not the writer's layout
    pkg.tdp.Tile(pctx, shuffled).free()
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(shuffled), attach=True)
    assert e.value.code == 4


def test_attach_reports_content_errors_like_the_host_parser(pkg, pctx):
    """The attach's metadata pass runs on the GPU; a voxel table it finds
    wrong sends the tile to the host parser, so the error is the one a
    sequential read meets first, with the host parser's message."""
    import struct
    from test_raw_parse import corrupt_box
    nb, _ = pkg.tdp.gen_tiles(10, 200, seed=5)
    off = pkg.tdp.raw_object_offsets(nb)
    for bad in ([7], [1500, 40]):
        b = nb
        for o in bad:
            b = corrupt_box(b, off, o)
        with pytest.raises(pkg.TdpError) as e:
            pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(b), attach=True)
        assert e.value.code == 4
        assert str(e.value).endswith("inverted voxel box in object %d" % min(bad))
    b = nb.copy()
    p = int(off[321])
    (ds,) = struct.unpack_from("<Q", b, p)
    struct.pack_into("<Q", b, p + 8 + ds + 8 + 40 + 36, ds + 4)  # first voxel's LOD-20 offset past the data block
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(b), attach=True)
    assert str(e.value).endswith("voxel lod range outside data block in object 321")


def test_attached_metadata_equal_uploaded(pkg, pctx):
    """Counts, boxes and transforms the GPU pass derives equal the host parser's."""
    nb, vb = tiles(8, 10, 104)
    for raw in (nb, vb):
        U = pkg.tdp.Tile(pctx, raw)
        A = pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(raw), attach=True)
        iu, ia = U.info(), A.info()
        for k in ("n_objects", "n_voxels", "n_tris"):
            assert iu[k] == ia[k], k
        assert ia["attached"] == 1
        # the GPU candidates read the attached tile's boxes and transforms
        for kw in (dict(knn=3), dict(within=200.0)):
            o1, i1 = pkg.tdp.tile_candidates(pctx, U, None, **kw)
            o2, i2 = pkg.tdp.tile_candidates(pctx, A, None, **kw)
            np.testing.assert_array_equal(o1, o2)
            np.testing.assert_array_equal(i1, i2)
        U.free()
        A.free()


def test_strided_attach_equals_walked(pkg, pctx):
    """A tile of equal-size records is attached without a host walk (records
    placed at the first record's stride, every object's size fields checked
    on the GPU).  Records of equal size but different kinds (1 voxel with
    triangles, or 12 voxels without) fail that check at the first record of
    the other kind and the tile is walked on the host: both give the host
    parser's counts and, for the generated tile, the uploaded tile's
    candidates."""
    from test_raw_parse import _uniform_tile, _record
    nb, _ = pkg.tdp.gen_tiles(10, 200, seed=9)           # 2,000 equal nucleus records: strided
    U = pkg.tdp.Tile(pctx, nb)
    A = pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(nb), attach=True)
    for k in ("n_objects", "n_voxels", "n_tris"):
        assert U.info()[k] == A.info()[k], k
    o1, i1 = pkg.tdp.tile_candidates(pctx, U, None, knn=4)
    o2, i2 = pkg.tdp.tile_candidates(pctx, A, None, knn=4)
    np.testing.assert_array_equal(o1, o2)
    np.testing.assert_array_equal(i1, i2)
    U.free()
    A.free()
    raw, nvox, _ = _uniform_tile(3000, 12)               # two record kinds of one size: walked after the check
    assert len(_record("A")) == len(_record("B"))
    A = pkg.tdp.Tile(pctx, pkg.tdp.pinned_copy(raw), attach=True)
    info = A.info()
    assert info["n_objects"] == 3000 and info["n_voxels"] == int(nvox.sum())
    A.free()
