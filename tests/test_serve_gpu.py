"""Serving (tdp_server_*): requests with different queries, batched together
by the continuous-batching loop, each get exactly the result of a join of that
request alone."""
import threading

import numpy as np
import pytest

from join_cases import tiles
from rawdt import read_tile, write_tile

pytestmark = pytest.mark.gpu

NV, NPV, SEED = 6, 12, 101
# (nuclei range, query, K, tau)
REQUESTS = [((0, 5), "nn", 3, 0.0), ((5, 17), "within", 0, 150.0), ((17, 18), "nn", 1, 0.0),
            ((18, 40), "nn", 5, 0.0), ((40, 47), "within", 0, 60.0), ((47, 72), "within", 0, 400.0),
            ((10, 30), "nn", 2, 0.0), ((36, 72), "within", 0, 100.0)]


@pytest.fixture(scope="module")
def setup(pkg, ctx):
    _, vb = tiles(NV, NPV, SEED)
    T2 = pkg.tdp.Tile(ctx, vb)
    reqs = []
    for (b, e), query, K, tau in REQUESTS:
        nb, _ = pkg.tdp.gen_tiles(NV, NPV, seed=SEED, nuclei_begin=b, nuclei_end=e)
        reqs.append((np.array(nb), query, K, tau))
    alone = []
    for raw, query, K, tau in reqs:
        T1 = pkg.tdp.Tile(ctx, raw)
        alone.append(ctx.join(T1, T2, query=query, knn=max(K, 1), within=tau))
        T1.free()
    return T2, reqs, alone


@pytest.mark.parametrize("arena_objects", [40, 100000])
@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("big_ms", [4.0, 0.005])
def test_each_request_equals_its_join_alone(pkg, ctx, setup, arena_objects, pinned, big_ms):
    """pinned: requests in page-locked memory, whose triangles the batch joins
    fetch from the caller's bytes instead of staging them whole.  big_ms =
    0.005: these requests' estimated join times (3 of them below, 5 above)
    make every mixed batch run as a small pass then a big pass."""
    T2, reqs, alone = setup
    bufs = [pkg.tdp.pinned_copy(r[0]) if pinned else r[0] for r in reqs]
    with pkg.tdp.Server(ctx, T2, arena_objects=arena_objects, arena_voxels=1 << 16, arena_tris=1 << 20,
                        max_request_bytes=64 << 20, big_request_ms=big_ms) as srv:
        ids = [None] * len(reqs)

        def client(k):
            _, query, K, tau = reqs[k]
            ids[k] = srv.submit(bufs[k], query=query, knn=max(K, 1), within=tau)

        threads = [threading.Thread(target=client, args=(k,)) for k in range(len(reqs))]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        infos = []
        for k, rid in enumerate(ids):
            q, t, d, info = srv.wait(rid, timeout_ms=60000)
            aq, at, ad = alone[k]
            np.testing.assert_array_equal(q, aq)
            np.testing.assert_array_equal(t, at)
            np.testing.assert_array_equal(d, ad)
            assert info["latency_ms"] >= info["queue_ms"] >= 0.0
            infos.append(info)
        st = srv.stats()
        assert st["requests"] == len(reqs) and st["failed"] == 0
        raw_bytes = sum(r[0].size for r in reqs)
        if pinned:
            assert 0 < st["fetch_bytes"] < raw_bytes and st["upload_bytes"] < raw_bytes / 4, st
        else:
            assert st["fetch_bytes"] == 0 and st["upload_bytes"] >= raw_bytes / 2, st
        if arena_objects == 40:
            assert st["batches"] >= 4  # 128 objects of requests, at most 40 per batch
        assert max(i["batch_requests"] for i in infos) >= 2  # requests were mixed in a batch
        if big_ms == 4.0:
            assert st["split_batches"] == 0  # every request here is far below 4 ms
        elif arena_objects == 100000 and max(i["batch_requests"] for i in infos) == len(reqs):
            assert st["split_batches"] >= 1  # one batch held small and big requests
    # the context is usable again after the server is closed
    raw, query, K, tau = reqs[0]
    T1 = pkg.tdp.Tile(ctx, raw)
    q, t, d = ctx.join(T1, T2, query=query, knn=max(K, 1), within=tau)
    np.testing.assert_array_equal(q, alone[0][0])
    T1.free()


def test_rejected_requests(pkg, ctx, setup):
    T2, reqs, _ = setup
    with pkg.tdp.Server(ctx, T2, arena_objects=10, arena_voxels=1 << 12, arena_tris=1 << 16,
                        max_request_bytes=64 << 20) as srv:
        with pytest.raises(pkg.TdpError):  # 36 objects > a 10-object arena
            srv.submit(reqs[-1][0], query="within", within=100.0)
        with pytest.raises(pkg.TdpError):  # malformed bytes
            srv.submit(np.zeros(64, np.uint8), query="nn", knn=1)
        with pytest.raises(pkg.TdpError):  # bad query
            srv.submit(reqs[0][0], query="nn", knn=0)
        rid = srv.submit(reqs[0][0], query="nn", knn=3)
        q, t, d, _ = srv.wait(rid)
        assert len(q) == 3 * 5


def test_page_locked_request_outside_the_writer_layout_is_staged(pkg, ctx, setup):
    """A page-locked request whose objects keep their LOD blocks in another
    order cannot be fetched (the fetch computes offsets in the writer's
    layout): the server stages its triangles, and the result equals the same
    objects in the writer's layout, which are fetched."""
    T2, reqs, _ = setup
    objs = [[list(o.tris[li]) for li in range(5)] for o in read_tile(reqs[5][0])]
    canonical = pkg.tdp.pinned_copy(write_tile(objs))
    shuffled = pkg.tdp.pinned_copy(write_tile(objs, lod_order=(4, 3, 2, 1, 0)))
    out = []
    for raw in (canonical, shuffled):
        with pkg.tdp.Server(ctx, T2, arena_objects=100, arena_voxels=1 << 16, arena_tris=1 << 20,
                            max_request_bytes=64 << 20) as srv:
            rid = srv.submit(raw, query="within", within=400.0)
            out.append(srv.wait(rid, timeout_ms=60000)[:3])
            out.append(srv.stats())
    (a, st_a, b, st_b) = out
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    assert len(a[0]) > 0
    # the fetched request sends only its metadata; the staged one its triangles too
    assert st_a["upload_bytes"] < canonical.size / 4, st_a
    assert st_b["fetch_bytes"] == 0 and st_b["upload_bytes"] >= shuffled.size / 2, st_b
