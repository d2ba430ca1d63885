"""A join split into query ranges by the product's partitioner and joined
range by range on the GPU (tdp_join_params.query_begin / query_end, the way
each rank of a multi-GPU run joins its shard) gives, concatenated, exactly
the whole join -- within, kNN and a kNN self-join, both forms -- and a
range join reports only queries inside its range.  One GPU runs the shards
one after another; the shards share nothing but tile 2, so running them on
separate GPUs changes only where they run."""
import numpy as np
import pytest

from join_cases import tiles

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shard_tiles(pkg, ctx):
    nb, vb = tiles(6, 12, 101)
    T1, T2 = pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb)
    yield nb, vb, T1, T2
    T1.free()
    T2.free()


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("kw", [dict(query="within", within=150.0), dict(query="nn", knn=3),
                                dict(query="nn", knn=4, self_join=True)])
@pytest.mark.parametrize("n_shards", [2, 3, 7])
def test_shards_concatenate_to_the_whole_join(pkg, ctx, shard_tiles, form, kw, n_shards):
    nb, vb, T1, T2 = shard_tiles
    kw = dict(kw)
    self_join = kw.pop("self_join", False)
    t2, raw2 = (None, None) if self_join else (T2, vb)
    whole = ctx.join(T1, t2, form=form, **kw)
    bounds, _ = pkg.shard.partition(nb, raw2, n_shards, knn=kw.get("knn", 0) if kw["query"] == "nn" else 0,
                                    within=kw.get("within", 0.0))
    parts = []
    for s in range(n_shards):
        b, e = pkg.shard.shard_range(bounds, s)
        q, t, d = ctx.join(T1, t2, form=form, query_range=(b, e), **kw)
        assert q.size == 0 or (q.min() >= b and q.max() < e)
        parts.append((q, t, d))
    gq, gt, gd = pkg.shard.merge_results(parts)
    np.testing.assert_array_equal(gq, whole[0])
    np.testing.assert_array_equal(gt, whole[1])
    np.testing.assert_array_equal(gd, whole[2].astype(np.float64))


def test_bad_query_ranges_are_errors(pkg, ctx, shard_tiles):
    _, _, T1, T2 = shard_tiles
    for r in ((-1, 3), (5, 2), (0, 73)):
        with pytest.raises(pkg.TdpError):
            ctx.join(T1, T2, query="nn", knn=2, query_range=r)
    q, _, _ = ctx.join(T1, T2, query="nn", knn=2, query_range=(10, 10))
    assert q.size == 0
