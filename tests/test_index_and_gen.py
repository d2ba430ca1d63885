"""CPU tests: tile generator + RAW format, object candidates, CPU join checkers."""
import hashlib

import numpy as np
import pytest

from join_cases import CASES, exact_truth, tiles
from oracle_bind import oracle, ref_join, reference
from rawdt import read_tile


def test_generator_is_deterministic_and_well_formed(pkg):
    nb, vb = pkg.tdp.gen_tiles(3, 4, seed=5)
    nb2, vb2 = pkg.tdp.gen_tiles(3, 4, seed=5)
    assert hashlib.sha256(nb.tobytes()).hexdigest() == hashlib.sha256(nb2.tobytes()).hexdigest()
    assert hashlib.sha256(vb.tobytes()).hexdigest() == hashlib.sha256(vb2.tobytes()).hexdigest()
    N, V = read_tile(nb), read_tile(vb)
    assert len(N) == 12 and len(V) == 3
    for o in N:
        assert [len(o.lod_tris(l)) for l in range(5)] == [256, 512, 768, 1024, 1280]
        assert len(o.voxels) == 13
        assert o.hausdorff[4] == 0 and o.proxyhausdorff[4] == 0
    for o in V:
        assert abs(len(o.lod_tris(4)) - 20000) < 500
        assert 150 <= len(o.voxels) <= 210
    for o in N + V:
        # every triangle of a voxel, at every LOD, lies inside the voxel box
        for l in range(5):
            for v, t in enumerate(o.tris[l]):
                if len(t):
                    p = t.reshape(-1, 3)
                    assert (p >= o.voxels[v, :3]).all() and (p <= o.voxels[v, 3:6]).all()
        # cores and transforms are surface points (mesh vertices)
        allv = o.lod_tris(4).reshape(-1, 3)
        assert (np.abs(allv - o.transform).sum(1) == 0).any()
        for c in o.voxels[:, 6:9]:
            assert (np.abs(allv - c).sum(1) == 0).any()


def test_generator_nuclei_do_not_touch(pkg):
    nb, vb = tiles(4, 16, 105)
    N = read_tile(nb)
    c = np.stack([o.box[:3] + o.box[3:] for o in N]) / 2
    d = np.linalg.norm(c[:, None] - c[None], axis=-1) + np.eye(len(c)) * 1e9
    assert d.min() > 2 * 13.2


def test_hausdorff_bounds_are_conservative(pkg):
    """d_LOD - ph1 - ph2 <= d_100 <= d_LOD + h1 + h2 for two whole objects (FP64 oracle)."""
    nb, vb = pkg.tdp.gen_tiles(1, 3, seed=11)
    N = read_tile(nb)
    O = oracle()
    a, b = N[0], N[1]
    d100 = O.voxel_pair(a.lod_tris(4), None, b.lod_tris(4), None)[0]
    for l in range(4):
        ha = np.concatenate(a.hds[l])
        hb = np.concatenate(b.hds[l])
        r = O.voxel_pair(a.lod_tris(l), ha, b.lod_tris(l), hb)
        assert r[1] <= d100 + 1e-9 <= r[2] + 2e-9, (l, r, d100)


def test_candidates_match_reference_octree(pkg, ref):
    if ref is None:
        pytest.skip("reference CPU code not built")
    nb, vb = tiles(6, 12, 101)
    N, V = read_tile(nb), read_tile(vb)
    b1 = np.stack([o.box for o in N]); x1 = np.stack([o.transform for o in N])
    b2 = np.stack([o.box for o in V]); x2 = np.stack([o.transform for o in V])
    for args in [dict(knn=3), dict(knn=1), dict(within=150.0), dict(within=400.0)]:
        off, ids = pkg.tdp.candidates(b1, x1, b2, x2, **args)
        roff, rids = ref.candidates(b1, x1, b2, x2, False, args.get("knn", 1), args.get("within", 0.0),
                                    "knn" in args)
        np.testing.assert_array_equal(off, roff)
        np.testing.assert_array_equal(ids, rids)
    for args in [dict(knn=5), dict(within=60.0)]:
        off, ids = pkg.tdp.candidates(b1, x1, b1, x1, self_join=True, **args)
        roff, rids = ref.candidates(b1, x1, b1, x1, True, args.get("knn", 1), args.get("within", 0.0),
                                    "knn" in args)
        np.testing.assert_array_equal(off, roff)
        np.testing.assert_array_equal(ids, rids)


def test_candidates_edge_cases(pkg):
    b = np.array([[0, 0, 0, 1, 1, 1]], np.float32)
    x = np.array([[0.5, 0.5, 0.5]], np.float32)
    off, ids = pkg.tdp.candidates(b, x, b, x, self_join=True, knn=3)
    assert off.tolist() == [0, 0] and len(ids) == 0
    off, ids = pkg.tdp.candidates(b, x, b, x, knn=3)
    assert ids.tolist() == [0]
    e = np.zeros((0, 6), np.float32)
    off, ids = pkg.tdp.candidates(e, np.zeros((0, 3), np.float32), b, x, within=5.0)
    assert off.tolist() == [0]


@pytest.mark.parametrize("name", ["knn3_nuc_ves", "within150", "knn5_self"])
def test_reference_rules_agree_with_exact_oracle(name):
    if reference() is None:
        pytest.skip("reference CPU code not built")
    nv, npv, seed, query, knn, tau, self_join, lods, level = CASES[name]
    nb, vb = tiles(nv, npv, seed)
    rq, rt, st = ref_join(nb, None if self_join else vb, self_join, query == "nn", knn=knn, tau=tau)
    truth, margin = exact_truth(nb, vb, self_join, query, knn, tau)
    assert margin > 1e-3
    assert set(zip(rq.tolist(), rt.tolist())) == truth


def _overlapping_nuclei(pkg):
    """Two nuclei tiles of different seeds around the same vessel grid, in a
    tight shell, so that many nuclei boxes (and some nuclei) overlap."""
    a, _ = pkg.tdp.gen_tiles(3, 100, seed=301, shell_min=12.0, shell_max=30.0)
    b, _ = pkg.tdp.gen_tiles(3, 100, seed=302, shell_min=12.0, shell_max=30.0)
    return a, b


def test_intersect_candidates_match_reference_octree(pkg, ref):
    """Intersect candidates (strict box overlap, OctreeNode::query_intersect)
    equal the reference octree's, compiled from source, set and order."""
    if ref is None:
        pytest.skip("reference CPU code not built")
    a, b = _overlapping_nuclei(pkg)
    A, B = read_tile(a), read_tile(b)
    b1 = np.stack([o.box for o in A]); x1 = np.stack([o.transform for o in A])
    b2 = np.stack([o.box for o in B]); x2 = np.stack([o.transform for o in B])
    off, ids = pkg.tdp.candidates(b1, x1, b2, x2, intersect=True)
    roff, rids = ref.candidates(b1, x1, b2, x2, False, 1, 0.0, 2)
    np.testing.assert_array_equal(off, roff)
    np.testing.assert_array_equal(ids, rids)
    assert len(ids) >= 10
    off, ids = pkg.tdp.candidates(b1, x1, b1, x1, self_join=True, intersect=True)
    roff, rids = ref.candidates(b1, x1, b1, x1, True, 1, 0.0, 2)
    np.testing.assert_array_equal(off, roff)
    np.testing.assert_array_equal(ids, rids)
