"""Properties of the FP64 oracle that hold at any size, beside its pins to
the golden vectors: the triangle distance is symmetric and invariant under
rigid motions and vertex order, no sampled point pair of the two triangles
is closer (and dense samples come close), and a within join of two tiles is
the transpose of the join with the tiles swapped."""
import numpy as np
import pytest

from oracle_bind import join_exact


def _tris(rng, n, spread=3.0):
    """n random triangle pairs: sizes 0.1-3, offsets up to `spread`, some
    nearly parallel and some sharing a vertex"""
    S = rng.normal(size=(n, 3, 3)) * rng.uniform(0.1, 3.0, (n, 1, 1))
    T = rng.normal(size=(n, 3, 3)) * rng.uniform(0.1, 3.0, (n, 1, 1)) + rng.normal(size=(n, 1, 3)) * spread
    k = n // 8
    T[:k] = S[:k] + rng.normal(size=(k, 1, 3)) * 0.5 + rng.normal(size=(k, 3, 3)) * 1e-4   # near-parallel copies
    T[k:2 * k, 0] = S[k:2 * k, 1]                                                             # shared vertex
    return S.reshape(n, 9), T.reshape(n, 9)


def _rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q *= np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def test_symmetric(orc):
    rng = np.random.default_rng(1)
    S, T = _tris(rng, 2000)
    d1, f1 = orc.tri_dist_batch(S, T)
    d2, f2 = orc.tri_dist_batch(T, S)
    np.testing.assert_allclose(d1, d2, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(f1, f2, rtol=1e-12, atol=1e-12)


def test_rigid_motion_and_vertex_order(orc):
    rng = np.random.default_rng(2)
    S, T = _tris(rng, 2000)
    d, _ = orc.tri_dist_batch(S, T)
    R, t = _rotation(rng), rng.normal(size=3) * 50

    def move(X):
        return (X.reshape(-1, 3, 3) @ R.T + t).reshape(-1, 9)

    dm, _ = orc.tri_dist_batch(move(S), move(T))
    np.testing.assert_allclose(dm, d, rtol=1e-9, atol=1e-9)
    for perm in ((1, 2, 0), (2, 1, 0)):
        Sp = S.reshape(-1, 3, 3)[:, perm].reshape(-1, 9)
        Tp = T.reshape(-1, 3, 3)[:, perm[::-1]].reshape(-1, 9)
        dp, _ = orc.tri_dist_batch(Sp, Tp)
        np.testing.assert_allclose(dp, d, rtol=1e-12, atol=1e-12)


def test_no_sampled_pair_is_closer(orc):
    """Every pair of points sampled on the two triangles is at least the
    distance apart, and the closest of a dense barycentric grid is within the
    grid's spacing of it."""
    rng = np.random.default_rng(3)
    S, T = _tris(rng, 200)
    d, _ = orc.tri_dist_batch(S, T)
    m = 24
    u, v = np.meshgrid(np.arange(m + 1), np.arange(m + 1))
    keep = u + v <= m
    bary = np.stack([u[keep], v[keep], m - u[keep] - v[keep]], 1) / m          # [P, 3]
    for i in range(len(S)):
        A, B = S[i].reshape(3, 3), T[i].reshape(3, 3)
        pa, pb = bary @ A, bary @ B
        gap = np.sqrt(((pa[:, None, :] - pb[None, :, :]) ** 2).sum(-1)).min()
        assert gap >= d[i] - 1e-9 * (1 + np.abs(A).max() + np.abs(B).max()), i
        edge = max(np.linalg.norm(A[j] - A[(j + 1) % 3]) for j in range(3)) + \
            max(np.linalg.norm(B[j] - B[(j + 1) % 3]) for j in range(3))
        assert gap <= d[i] + edge / m + 1e-9, i


@pytest.mark.parametrize("tau", [60.0, 250.0])
def test_within_join_is_symmetric(pkg, tau):
    """within(A, B) holds (q, t) exactly when within(B, A) holds (t, q): the
    exact object distance does not depend on which tile is the query tile."""
    nb, vb = pkg.tdp.gen_tiles(2, 6, seed=17)
    q, t, _, hit = join_exact(nb, vb, False, False, tau=tau)
    q2, t2, _, hit2 = join_exact(vb, nb, False, False, tau=tau)
    a = set(zip(q[hit].tolist(), t[hit].tolist()))
    b = set(zip(t2[hit2].tolist(), q2[hit2].tolist()))
    assert a == b
    assert a, "the case should have results"
