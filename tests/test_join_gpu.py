"""End-to-end join parity on the GPU, through the C ABI.

For every seeded case, both forms (plain, tuned) must return exactly the result
set of (a) the reference's own join rules run on the CPU with the reference's
compiled FP32 MeshDist and octree (oracle/_ref) and (b) the FP64 exact oracle
(asserted only when the exact distances keep every decision at least 1e-3
away from a tie, which the generator's seeds guarantee for these cases).
Result sets are compared as sorted (query id, result id) pairs, the way the
reference's tools/evaluate.cpp compares result files.
"""
import numpy as np
import pytest

from join_cases import CASES, exact_truth, tiles
from oracle_bind import ref_join

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_tiles(pkg, ctx):
    cache = {}

    def get(nv, npv, seed):
        key = (nv, npv, seed)
        if key not in cache:
            nb, vb = tiles(nv, npv, seed)
            cache[key] = (pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb))
        return cache[key]
    return get


@pytest.mark.parametrize("name", list(CASES))
def test_join_matches_reference_and_oracle(pkg, ctx, gpu_tiles, name):
    nv, npv, seed, query, knn, tau, self_join, lods, level = CASES[name]
    nb, vb = tiles(nv, npv, seed)
    T1, T2 = gpu_tiles(nv, npv, seed)
    ref = ref_join(nb, None if self_join else vb, self_join, query == "nn", knn=knn, tau=tau, lods=lods, level=level)
    got = {}
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        q, t, d = ctx.join(T1, None if self_join else T2, query=query, knn=knn, within=tau, lods=lods,
                           hausdorff_level=level, form=form)
        assert np.all(np.diff(q) >= 0)
        got[form] = set(zip(q.tolist(), t.tolist()))
        st = ctx.stats()
        assert st["total_ms"] > 0
    assert got[pkg.FORM_PLAIN] == got[pkg.FORM_TUNED], name
    if ref is not None:
        rq, rt, _ = ref
        assert got[pkg.FORM_PLAIN] == set(zip(rq.tolist(), rt.tolist())), name
    if lods is None or lods[-1] == 100:
        truth, margin = exact_truth(nb, vb, self_join, query, knn, tau)
        if margin > 1e-3 and level != 1:
            assert got[pkg.FORM_TUNED] == truth, name
            if query == "nn":
                n_q = len(set(q for q, _ in truth))
                assert len(truth) == knn * n_q


def test_knn_reports_exactly_k(pkg, ctx, gpu_tiles):
    nv, npv, seed = 6, 12, 101
    T1, T2 = gpu_tiles(nv, npv, seed)
    for K in (1, 2, 4):
        q, t, _ = ctx.join(T1, T2, query="nn", knn=K)
        counts = np.bincount(q, minlength=nv * npv)
        assert (counts == min(K, nv)).all()


def test_within_self_join_is_symmetric(pkg, ctx, gpu_tiles):
    T1, _ = gpu_tiles(4, 16, 106)
    q, t, _ = ctx.join(T1, None, query="within", within=60.0)
    pairs = set(zip(q.tolist(), t.tolist()))
    assert pairs == {(b, a) for a, b in pairs}
    assert all(a != b for a, b in pairs)


def test_join_stats_and_repeatability(pkg, ctx, gpu_tiles):
    T1, T2 = gpu_tiles(8, 10, 104)
    a = ctx.join(T1, T2, query="within", within=400.0)
    s1 = ctx.stats()
    b = ctx.join(T1, T2, query="within", within=400.0)
    s2 = ctx.stats()
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert s1["tri_pairs"] == s2["tri_pairs"]
    assert s1["filter_pairs"] > 0


def test_bad_arguments_are_errors(pkg, ctx, gpu_tiles):
    T1, T2 = gpu_tiles(6, 12, 101)
    with pytest.raises(pkg.TdpError):
        ctx.join(T1, T2, query="nn", knn=0)
    with pytest.raises(pkg.TdpError):
        ctx.join(T1, T2, query="nn", knn=2, lods=[30])
    with pytest.raises(pkg.TdpError):
        pkg.tdp.Tile(ctx, np.zeros(10, np.uint8))
    with pytest.raises(pkg.TdpError):
        pkg.tdp.Tile(ctx, np.frombuffer(bytes([1]) + bytes(7), np.uint8))


def test_tile_info(pkg, ctx, gpu_tiles):
    T1, T2 = gpu_tiles(6, 12, 101)
    i = T1.info()
    assert i["n_objects"] == 72 and i["n_tris"][4] == 72 * 1280
    assert i["n_tris"][0] == 72 * 256
    assert T2.info()["n_objects"] == 6


def test_cli_matches_library(pkg, ctx, gpu_tiles, tmp_path):
    """`tdbase join ... --print_result` prints the same pairs the C ABI returns."""
    import subprocess
    from pathlib import Path
    nb, vb = tiles(6, 12, 103)
    p1, p2 = tmp_path / "n.dt", tmp_path / "v.dt"
    nb.tofile(p1)
    vb.tofile(p2)
    exe = Path(pkg.__file__).parent / "bin" / "tdbase"
    out = subprocess.run([str(exe), "join", "--tile1", str(p1), "--tile2", str(p2), "-q", "within",
                          "--within_dist", "150", "--print_result", "-g"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    got = {tuple(map(int, l.split())) for l in out.stdout.splitlines() if l.strip()}
    T1, T2 = gpu_tiles(6, 12, 103)
    q, t, _ = ctx.join(T1, T2, query="within", within=150.0)
    assert got == set(zip(q.tolist(), t.tolist()))
    assert "results:" in out.stderr


@pytest.mark.parametrize("args", [dict(knn=3), dict(knn=1), dict(knn=7), dict(within=150.0), dict(within=400.0)])
def test_gpu_candidates_match_reference_octree(pkg, ctx, gpu_tiles, ref, args):
    """The GPU candidate generation (used by the tuned join) returns the reference
    octree's candidates, same set and same order, and agrees with the host grid."""
    from rawdt import read_tile
    nb, vb = tiles(6, 12, 101)
    T1, T2 = gpu_tiles(6, 12, 101)
    off, ids = pkg.tdp.tile_candidates(ctx, T1, T2, **args)
    N, V = read_tile(nb), read_tile(vb)
    b1 = np.stack([o.box for o in N]); x1 = np.stack([o.transform for o in N])
    b2 = np.stack([o.box for o in V]); x2 = np.stack([o.transform for o in V])
    hoff, hids = pkg.tdp.candidates(b1, x1, b2, x2, **args)
    np.testing.assert_array_equal(off, hoff)
    np.testing.assert_array_equal(ids, hids)
    if ref is not None:
        roff, rids = ref.candidates(b1, x1, b2, x2, False, args.get("knn", 1), args.get("within", 0.0), "knn" in args)
        np.testing.assert_array_equal(off, roff)
        np.testing.assert_array_equal(ids, rids)


@pytest.mark.parametrize("args", [dict(knn=5), dict(within=60.0)])
def test_gpu_candidates_self_join(pkg, ctx, gpu_tiles, ref, args):
    from rawdt import read_tile
    nb, _ = tiles(4, 16, 105)
    T1, _ = gpu_tiles(4, 16, 105)
    off, ids = pkg.tdp.tile_candidates(ctx, T1, None, **args)
    N = read_tile(nb)
    b1 = np.stack([o.box for o in N]); x1 = np.stack([o.transform for o in N])
    hoff, hids = pkg.tdp.candidates(b1, x1, b1, x1, self_join=True, **args)
    np.testing.assert_array_equal(off, hoff)
    np.testing.assert_array_equal(ids, hids)


def test_refine_configs_identical_and_autotune(pkg, ctx, gpu_tiles):
    """Every tuned-refine configuration returns bit-identical joins; the
    autotuner times them all and keeps a valid one for the context."""
    T1, T2 = gpu_tiles(6, 12, 101)
    cfgs = pkg.tdp.refine_configs()
    assert len(cfgs) >= 2 and all(a % 8 == 0 and c >= 1 for a, c in cfgs)
    keep = ctx.refine_config()
    queries = (dict(query="within", within=150.0), dict(query="nn", knn=3))
    first = []
    try:
        for args in queries:
            outs = []
            for c in range(len(cfgs)):
                ctx.set_refine_config(c)
                outs.append(ctx.join(T1, T2, form=pkg.FORM_TUNED, **args))
            for o in outs[1:]:
                for a, b in zip(outs[0], o):
                    np.testing.assert_array_equal(a, b)
            first.append(outs[0])
        best, ms = ctx.autotune(T1, T2, query="within", within=150.0)
        assert 0 <= best < len(cfgs) and ctx.refine_config() == best
        assert len(ms) == len(cfgs) and all(m > 0 for m in ms)
        # each LOD runs the configuration fastest at that LOD; results unchanged
        by_lod = ctx.refine_configs_by_lod()
        assert sorted(by_lod) == [20, 40, 60, 80, 100] and all(0 <= c < len(cfgs) for c in by_lod.values())
        for args, want in zip(queries, first):
            for a, b in zip(ctx.join(T1, T2, form=pkg.FORM_TUNED, **args), want):
                np.testing.assert_array_equal(a, b)
        ctx.set_refine_config(0)
        assert set(ctx.refine_configs_by_lod().values()) == {0}
        with pytest.raises(pkg.TdpError):
            ctx.set_refine_config(len(cfgs))
    finally:
        ctx.set_refine_config(keep)


@pytest.mark.parametrize("name", list(CASES))
def test_exact_distances_match_fp64_oracle(pkg, ctx, gpu_tiles, name):
    """With exact_distances every result carries its LOD-100 distance in FP64:
    within 1e-9 relative of the FP64 oracle's exact object distance."""
    from oracle_bind import join_exact
    nv, npv, seed, query, knn, tau, self_join, lods, level = CASES[name]
    nb, vb = tiles(nv, npv, seed)
    T1, T2 = gpu_tiles(nv, npv, seed)
    oq, ot, od, _ = join_exact(nb, None if self_join else vb, self_join, query == "nn", knn=knn, tau=tau)
    truth = {(int(a), int(b)): float(x) for a, b, x in zip(oq, ot, od)}
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        q, t, d = ctx.join(T1, None if self_join else T2, query=query, knn=knn, within=tau, lods=lods,
                           hausdorff_level=level, form=form, exact_distances=True)
        assert d.dtype == np.float64 and len(d) == len(q) > 0
        ref = np.array([truth[(int(a), int(b))] for a, b in zip(q, t)])
        err = np.abs(d - ref) / np.maximum(ref, 1.0)
        assert err.max() <= 1e-9, (name, form, float(err.max()))
        st = ctx.stats()
        assert st["exact_items"] >= len(q) and 0 < st["exact_f64_items"] <= st["exact_items"]
        # the FP32 refine's own error against FP64 stays far inside its 64uR model
        assert 0.0 <= st["fp32_max_rel_err"] < 1e-4
        # the ids are those of the join without the exact stage
        q2, t2, d2 = ctx.join(T1, None if self_join else T2, query=query, knn=knn, within=tau, lods=lods,
                              hausdorff_level=level, form=form)
        np.testing.assert_array_equal(q, q2)
        np.testing.assert_array_equal(t, t2)
        assert d2.dtype == np.float32
        # at Hausdorff level 2 every FP32 result distance is an upper bound of
        # the exact one (within its error band)
        if level == 2:
            assert np.all(d2.astype(np.float64) >= d * (1 - 1e-5) - 1e-4)


def test_mixed_queries_equal_separate_joins(pkg, ctx, gpu_tiles):
    """One join whose query objects carry different queries (kNN with several
    K, within with several tau) returns, for every object, exactly what a join
    of that object's own query returns: same ids, same distances."""
    nb, vb = tiles(6, 12, 101)
    T1, T2 = gpu_tiles(6, 12, 101)
    n1 = T1.info()["n_objects"]
    specs = [("nn", 1, 0.0), ("nn", 3, 0.0), ("nn", 5, 0.0), ("within", 0, 60.0), ("within", 0, 150.0)]
    rng = np.random.default_rng(7)
    which = rng.integers(0, len(specs), n1)
    ok = np.array([specs[w][1] for w in which], np.int32)
    ow = np.array([specs[w][2] for w in which], np.float32)
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        q, t, d = ctx.join(T1, T2, form=form, obj_knn=ok, obj_within=ow)
        want_q, want_t, want_d = [], [], []
        for k, (query, K, tau) in enumerate(specs):
            aq, at, ad = ctx.join(T1, T2, query=query, knn=max(K, 1), within=tau, form=form)
            m = which[aq] == k
            want_q.append(aq[m]); want_t.append(at[m]); want_d.append(ad[m])
        wq, wt, wd = (np.concatenate(x) for x in (want_q, want_t, want_d))
        o = np.lexsort((wt, wq))
        np.testing.assert_array_equal(q, wq[o])
        np.testing.assert_array_equal(t, wt[o])
        np.testing.assert_array_equal(d, wd[o])
        # every kNN object reports exactly its own K
        for k, (query, K, tau) in enumerate(specs):
            if query == "nn":
                objs = np.nonzero(which == k)[0]
                counts = np.bincount(q, minlength=n1)[objs]
                assert np.all(counts == K)


def test_lod_graph_modes_identical(pkg):
    """The tuned LOD loop launched directly, captured as a CUDA graph, and
    replayed from the graph returns the same ids and distances.  Auto mode
    launches new arguments directly, captures them on their second use and
    replays them after that; a change of arguments (query, distance, LOD list,
    self-join) captures or updates the graph again; the per-LOD refine timing
    still works in a replay.  A join whose filter decides every pair has no
    LOD loop (no refine launch) and so no graph."""
    c = pkg.Context(0)
    try:
        nb, vb = tiles(6, 12, 101)
        T1, T2 = pkg.tdp.Tile(c, nb), pkg.tdp.Tile(c, vb)
        runs = [(T2, dict(query="nn", knn=3)), (T2, dict(query="within", within=150.0)),
                (T2, dict(query="nn", knn=1, lods=[40, 100])), (T2, dict(query="within", within=60.0, lods=[40, 100])),
                (T2, dict(query="nn", knn=2, lods=[20, 60, 100])), (None, dict(query="within", within=60.0)),
                (None, dict(query="nn", knn=4)), (T2, dict(query="nn", knn=3, lods=[20, 40]))]
        want, looped = {}, {}
        for i, (t2, args) in enumerate(runs):
            nl = len(args.get("lods") or [20, 40, 60, 80, 100])
            c.set_lod_graph(pkg.tdp.LOD_GRAPH_OFF)
            want[i] = c.join(T1, t2, **args)
            st = c.stats()
            assert st["lod_graph"] == 0
            looped[i] = st["refine_launches"] > 0
            c.set_lod_graph(pkg.tdp.LOD_GRAPH_AUTO)
            how = []
            for _ in range(3):
                got = c.join(T1, t2, **args)
                st = c.stats()
                how.append(st["lod_graph"])
                assert st["refine_launches"] == (nl if looped[i] else 0)
                if looped[i]:
                    assert st["refine_ms"] > 0
                for a, b in zip(got, want[i]):
                    np.testing.assert_array_equal(a, b)
            assert how == ([0, 2, 1] if looped[i] else [0, 0, 0]), (args, how)
        assert sum(looped.values()) >= 4
        c.set_lod_graph(pkg.tdp.LOD_GRAPH_ALWAYS)
        for i, (t2, args) in enumerate(runs):
            for expect in ((2, 1) if looped[i] else (0, 0)):
                got = c.join(T1, t2, **args)
                assert c.stats()["lod_graph"] == expect
                for a, b in zip(got, want[i]):
                    np.testing.assert_array_equal(a, b)
        with pytest.raises(pkg.TdpError):
            c.set_lod_graph(3)
        T1.free()
        T2.free()
    finally:
        c.close()


def test_intersect_join_matches_fp64_truth(pkg, ctx):
    """-q intersect: the pairs whose boxes overlap strictly and whose LOD-100
    meshes touch or cross (exact FP64 distance 0); both forms."""
    from oracle_bind import join_exact
    from rawdt import read_tile
    a, _ = pkg.tdp.gen_tiles(3, 100, seed=301, shell_min=12.0, shell_max=30.0)
    b, _ = pkg.tdp.gen_tiles(3, 100, seed=302, shell_min=12.0, shell_max=30.0)
    oq, ot, od, _ = join_exact(a, b, False, False, tau=0.0)
    A, B = read_tile(a), read_tile(b)

    def strict(x, y):
        return not any(y[i] >= x[i + 3] or y[i + 3] <= x[i] for i in range(3))

    truth = {(int(q), int(t)) for q, t, d in zip(oq, ot, od) if d == 0.0 and strict(A[q].box, B[t].box)}
    assert len(truth) > 0
    T1, T2 = pkg.tdp.Tile(ctx, a), pkg.tdp.Tile(ctx, b)
    for form in (pkg.FORM_PLAIN, pkg.FORM_TUNED):
        q, t, d = ctx.join(T1, T2, query="intersect", form=form)
        assert set(zip(q.tolist(), t.tolist())) == truth, form
        assert np.all(d == 0.0)


@pytest.mark.parametrize("args", [dict(query="nn", knn=3), dict(query="within", within=150.0)])
@pytest.mark.parametrize("chunk", [1, 7, 1000])
def test_chunked_join_equals_whole_join(pkg, ctx, gpu_tiles, args, chunk):
    """tdp_join_chunked (tiles in host memory, tile 1 in chunks against
    sub-tiles of tile 2) returns the whole join's result, ids and distances."""
    nb, vb = tiles(6, 12, 101)
    T1, T2 = gpu_tiles(6, 12, 101)
    q, t, d = ctx.join(T1, T2, **args)
    cq, ct, cd, info = ctx.join_chunked(nb, vb, chunk, **args)
    np.testing.assert_array_equal(cq, q)
    np.testing.assert_array_equal(ct, t)
    np.testing.assert_array_equal(cd, d)
    assert info["chunks"] == -(-T1.info()["n_objects"] // chunk) and info["splits"] == 0


def test_chunked_join_fits_a_budget_the_whole_join_exceeds(pkg):
    """Config 4 in small: under a device budget below the two tiles' size the
    whole join fails with TDP_ERR_NOMEM; the chunked join succeeds within the
    same budget (a fresh context: the failed upload may keep scratch)."""
    nb, vb = tiles(2, 60, 107)
    budget = int(0.7 * (nb.size + vb.size))
    assert nb.size > budget  # the query tile alone does not fit
    with pkg.Context(0, budget) as small:
        with pytest.raises(pkg.TdpError) as e:
            pkg.tdp.Tile(small, nb)
        assert e.value.code == 3
    with pkg.Context(0, budget) as small:
        q, t, d, info = small.join_chunked(nb, vb, 1 << 30, query="nn", knn=2)  # chunks cut by the budget
        assert info["device_peak_bytes"] <= budget and info["chunks"] >= 2
        assert len(q) == 2 * 120
    with pkg.Context(0) as big:
        wq, wt, wd = big.join(pkg.tdp.Tile(big, nb), pkg.tdp.Tile(big, vb), query="nn", knn=2)
    np.testing.assert_array_equal(q, wq)
    np.testing.assert_array_equal(t, wt)
    np.testing.assert_array_equal(d, wd)
