"""Refine kernels (plain and tuned forms) against the FP64 oracle, through the C ABI.

Tolerance: the FP32 forward-error model of the kernels,
|d32 - d64| <= 64 * 2^-24 * R, R = largest |coordinate| after translating to the
voxel pair's origin (the first vertex of the A-side voxel), plus one rounding of
the Hausdorff additions for the two bounds.
"""
import numpy as np
import pytest

from oracle_bind import oracle

pytestmark = pytest.mark.gpu
U = 2.0 ** -24
ERR_C = 64.0
GOLD = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def make_batch(rng, n_pairs, sizes=(1, 90), gap=(0.0, 30.0), far=0.0):
    tris, hds, osz = [], [], []
    off = 0
    for k in range(n_pairs):
        n1 = int(rng.integers(sizes[0], sizes[1] + 1))
        n2 = int(rng.integers(sizes[0], sizes[1] + 1))
        base = rng.normal(size=3) * far
        g = rng.uniform(*gap)
        c1 = base + rng.normal(size=(n1, 3)) * 2.0
        c2 = base + np.array([g, 0.5, -0.3]) + rng.normal(size=(n2, 3)) * 2.0
        t1 = (c1[:, None, :] + rng.normal(size=(n1, 3, 3))).reshape(n1, 9)
        t2 = (c2[:, None, :] + rng.normal(size=(n2, 3, 3))).reshape(n2, 9)
        tris += [t1, t2]
        hds += [np.abs(rng.normal(size=(n1, 2))) * 0.3, np.abs(rng.normal(size=(n2, 2))) * 0.3]
        osz.append((off, n1, off + n1, n2))
        off += n1 + n2
    return (np.concatenate(tris).astype(np.float32), np.concatenate(hds).astype(np.float32),
            np.array(osz, np.uint64))


def oracle_batch(tri, hd, osz):
    O = oracle()
    return np.stack([O.voxel_pair(tri[o1:o1 + n1], None if hd is None else hd[o1:o1 + n1],
                                  tri[o2:o2 + n2], None if hd is None else hd[o2:o2 + n2])
                     for o1, n1, o2, n2 in osz.astype(np.int64)])


def local_scale(tri, osz):
    R = np.zeros(len(osz))
    for i, (o1, n1, o2, n2) in enumerate(osz.astype(np.int64)):
        if n1 == 0 or n2 == 0:
            continue
        o = tri[o1, :3].astype(np.float64)
        pts = np.concatenate([tri[o1:o1 + n1], tri[o2:o2 + n2]]).reshape(-1, 3).astype(np.float64)
        R[i] = np.abs(pts - o).max()
    return R


def check(got, want, tri, hd, osz):
    R = local_scale(tri, osz)
    tol = ERR_C * U * np.maximum(R, 1e-30)
    err = np.abs(got[:, 0].astype(np.float64) - want[:, 0])
    ratio = (err / (U * np.maximum(R, 1e-30))).max()
    assert (err <= tol).all(), f"distance error {err.max()} > tol; worst ratio {ratio}"
    if hd is not None:
        hmax = np.abs(hd).max() * 2 + 1
        tol2 = tol + 4 * U * (want[:, 2] + hmax)
        assert (np.abs(got[:, 1] - want[:, 1]) <= tol2).all()
        assert (np.abs(got[:, 2] - want[:, 2]) <= tol2).all()
    return ratio


@pytest.mark.parametrize("form", [0, 1])
def test_refine_random_voxel_pairs(ctx, form):
    rng = np.random.default_rng(7 + form)
    tri, hd, osz = make_batch(rng, 160)
    got = ctx.refine_batch(tri, hd, osz, form=form)
    want = oracle_batch(tri, hd, osz)
    ratio = check(got, want, tri, hd, osz)
    print(f"form {form}: worst |d32-d64|/(u R) = {ratio:.2f}")


@pytest.mark.parametrize("form", [0, 1])
def test_refine_far_from_origin(ctx, form):
    """Coordinates ~1e4 (a tile spans 10 vessel grid cells of 1000 units)."""
    rng = np.random.default_rng(11 + form)
    tri, hd, osz = make_batch(rng, 64, far=5000.0)
    got = ctx.refine_batch(tri, hd, osz, form=form)
    check(got, oracle_batch(tri, hd, osz), tri, hd, osz)


@pytest.mark.parametrize("form", [0, 1])
def test_refine_large_and_ragged(ctx, form):
    """Voxels larger than one shared-memory chunk (64 / 128 triangles), singletons."""
    rng = np.random.default_rng(3 + form)
    tri, hd, osz = make_batch(rng, 12, sizes=(1, 300))
    t1, h1, o1 = make_batch(rng, 8, sizes=(1, 1))
    osz2 = o1.copy()
    osz2[:, 0] += len(tri)
    osz2[:, 2] += len(tri)
    tri = np.concatenate([tri, t1])
    hd = np.concatenate([hd, h1])
    osz = np.concatenate([osz, osz2])
    got = ctx.refine_batch(tri, hd, osz, form=form)
    check(got, oracle_batch(tri, hd, osz), tri, hd, osz)


@pytest.mark.parametrize("form", [0, 1])
def test_refine_empty_side_and_no_hausdorff(ctx, form):
    rng = np.random.default_rng(5)
    tri, hd, osz = make_batch(rng, 6)
    osz[2, 1] = 0
    osz[4, 3] = 0
    got = ctx.refine_batch(tri, hd, osz, form=form)
    assert got[2, 0] == np.float32(3.4028235e38) and got[4, 0] == np.float32(3.4028235e38)
    got2 = ctx.refine_batch(tri, None, osz, form=form)
    assert (got2[:, 1:] == np.float32(3.4028235e38)).all()
    np.testing.assert_array_equal(got2[:, 0], got[:, 0])


@pytest.mark.parametrize("form", [0, 1])
def test_refine_touching_and_identical(ctx, form):
    rng = np.random.default_rng(9)
    tri, hd, osz = make_batch(rng, 20, gap=(0.0, 0.5))
    # identical voxel on both sides -> distance 0
    osz[0, 2] = osz[0, 0]
    osz[0, 3] = osz[0, 1]
    got = ctx.refine_batch(tri, hd, osz, form=form)
    want = oracle_batch(tri, hd, osz)
    assert got[0, 0] == 0.0
    check(got, want, tri, hd, osz)


def test_refine_matches_reference_meshdist_golden(ctx):
    m = np.load(GOLD / "meshdist_golden.npz")
    for form in (0, 1):
        got = ctx.refine_batch(m["tri"], m["hd"], m["offset_size"], form=form)
        check(got, m["oracle64"], m["tri"], m["hd"], m["offset_size"])
        np.testing.assert_allclose(got, m["ref32"], rtol=2e-6, atol=2e-5)


def test_plain_and_tuned_agree(ctx):
    rng = np.random.default_rng(21)
    tri, hd, osz = make_batch(rng, 300, sizes=(5, 120))
    a = ctx.refine_batch(tri, hd, osz, form=0)
    b = ctx.refine_batch(tri, hd, osz, form=1)
    R = local_scale(tri, osz)
    assert (np.abs(a[:, 0] - b[:, 0]) <= 2 * ERR_C * U * R).all()
    st = ctx.stats()
    assert st["full_evals"] <= st["tri_pairs"]


def test_tuned_configs_bit_identical(ctx, pkg):
    """The tuned kernel's configurations (A-chunk size, CTAs per SM) stage,
    translate and cull the same pairs conservatively: outputs are bit-identical,
    including voxels larger than every A chunk."""
    rng = np.random.default_rng(33)
    tri, hd, osz = make_batch(rng, 200, sizes=(1, 200))
    keep = ctx.refine_config()
    try:
        outs = []
        for c in range(len(pkg.tdp.refine_configs())):
            ctx.set_refine_config(c)
            outs.append(ctx.refine_batch(tri, hd, osz, form=1))
        for o in outs[1:]:
            np.testing.assert_array_equal(outs[0], o)
    finally:
        ctx.set_refine_config(keep)
