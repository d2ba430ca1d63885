"""kNN object candidates whose ring search outgrows a warp's shared-memory
buffer (1024 keys) stay on the GPU: the queries are redone there with a
global buffer, and the candidate lists still equal the host grid's and the
reference octree's (src/index/octree.cpp:215-291, compiled from source), the
same set in the same order.  A tuned join with such a K reports exactly K
results per query, equal to the reference's join rules, with its candidates
computed on the device.

K = 1030 is larger than the shared buffer, so every kNN query overflows it.
"""
import numpy as np
import pytest

from oracle_bind import ref_join

pytestmark = pytest.mark.gpu
K_BIG = 1030


@pytest.fixture(scope="module")
def dense(pkg, ctx):
    q_raw, _ = pkg.tdp.gen_tiles(1, 3, seed=4242)          # 3 query nuclei
    t_raw, _ = pkg.tdp.gen_tiles(11, 100, seed=4243)       # 1100 nuclei
    Q, T = pkg.tdp.Tile(ctx, q_raw), pkg.tdp.Tile(ctx, t_raw)
    yield q_raw, t_raw, Q, T
    Q.free()
    T.free()


def _boxes(raw):
    from rawdt import read_tile
    objs = read_tile(raw)
    return np.stack([o.box for o in objs]), np.stack([o.transform for o in objs])


def test_overflowing_candidates_match_host_and_reference(pkg, ctx, ref, dense):
    q_raw, t_raw, Q, T = dense
    off, ids = pkg.tdp.tile_candidates(ctx, Q, T, knn=K_BIG)
    assert ctx.stats()["candidate_redone"] == 3
    b1, x1 = _boxes(q_raw)
    b2, x2 = _boxes(t_raw)
    hoff, hids = pkg.tdp.candidates(b1, x1, b2, x2, knn=K_BIG)
    np.testing.assert_array_equal(off, hoff)
    np.testing.assert_array_equal(ids, hids)
    assert (np.diff(off) >= K_BIG).all()
    if ref is not None:
        roff, rids = ref.candidates(b1, x1, b2, x2, False, K_BIG, 0.0, True)
        np.testing.assert_array_equal(off, roff)
        np.testing.assert_array_equal(ids, rids)


def test_overflowing_self_join_candidates_match_host(pkg, ctx, dense):
    _, t_raw, _, T = dense
    off, ids = pkg.tdp.tile_candidates(ctx, T, None, knn=K_BIG)
    assert ctx.stats()["candidate_redone"] == 1100
    b, x = _boxes(t_raw)
    hoff, hids = pkg.tdp.candidates(b, x, b, x, self_join=True, knn=K_BIG)
    np.testing.assert_array_equal(off, hoff)
    np.testing.assert_array_equal(ids, hids)


def test_small_k_needs_no_second_pass(pkg, ctx, dense):
    _, _, Q, T = dense
    pkg.tdp.tile_candidates(ctx, Q, T, knn=5)
    assert ctx.stats()["candidate_redone"] == 0


def test_join_with_overflowing_candidates_stays_on_device(pkg, ctx, dense):
    q_raw, t_raw, Q, T = dense
    q, t, _ = ctx.join(Q, T, query="nn", knn=K_BIG, form=pkg.FORM_TUNED)
    st = ctx.stats()
    assert st["candidates_on_device"] == 1 and st["candidate_redone"] == 3
    assert (np.bincount(q, minlength=3) == K_BIG).all()
    got = set(zip(q.tolist(), t.tolist()))
    r = ref_join(q_raw, t_raw, False, True, knn=K_BIG)
    if r is not None:
        assert got == set(zip(r[0].tolist(), r[1].tolist()))
