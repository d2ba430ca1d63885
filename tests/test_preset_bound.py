"""The coordinate bound behind the last-LOD preset of a within item.

At the last LOD the tuned join refines each within item (a voxel pair)
against a preset of tau + 2 err_bound(R) + 1e-6, R = (tau + da + db) * 1.001
+ 1, where da and db are the L1 extents of the two voxels' boxes
(`within_preset`, 3dpipe_b200/csrc/join_kernels.cu).  An item with nothing
below the preset is then taken to have no triangle pair within tau.  That
holds because the FP32 error of a pair's distance is at most err_bound of its
largest coordinate, taken from the A voxel's first vertex, and every pair
within tau has all its coordinates below tau + da + db: an A vertex is in A's
box, and a B vertex is at most B's extent from the pair's closest B point,
which is within tau of the closest A point in A's box.  This test checks that
bound on random voxel pairs with the FP64 oracle's triangle distances,
including the pairs that come closest to it.
"""
import numpy as np

from oracle_bind import oracle


def _voxel(rng, n, centre, spread):
    """n triangles of size up to `spread` / 4 scattered over a patch of
    `spread` around `centre` (a voxel's triangles lie in its box)"""
    c = centre + rng.uniform(-spread, spread, size=(n, 1, 3))
    return (c + rng.normal(size=(n, 3, 3)) * spread / 8).reshape(n, 9)


def test_pairs_within_tau_stay_inside_the_preset_coordinate_bound():
    rng = np.random.default_rng(7)
    O = oracle()
    worst = 0.0
    checked = 0
    for trial in range(60):
        n1, n2 = rng.integers(4, 24, size=2)
        s1, s2 = rng.uniform(0.5, 40.0, size=2)
        gap = rng.uniform(0.0, 3.0) * (s1 + s2)
        A = _voxel(rng, n1, np.zeros(3), s1)
        B = _voxel(rng, n2, rng.normal(size=3) / np.sqrt(3) * gap, s2)
        # far from the origin too: the bound is on coordinates relative to o
        shift = rng.normal(size=3) * rng.choice([0.0, 1e3, 1e5])
        A = A + np.tile(shift, 3)
        B = B + np.tile(shift, 3)
        S = np.repeat(A, n2, axis=0)
        T = np.tile(B, (n1, 1))
        d, _ = O.tri_dist_batch(S, T)
        tau = float(np.quantile(d, rng.uniform(0.05, 0.6)))
        va, vb = A.reshape(-1, 3), B.reshape(-1, 3)
        da = float((va.max(0) - va.min(0)).sum())
        db = float((vb.max(0) - vb.min(0)).sum())
        o = A[0, :3]
        close = d <= tau
        assert close.any()
        coords = np.abs(np.concatenate([S[close], T[close]], axis=1).reshape(-1, 3) - o)
        # per axis, the exact statement: extent of A + tau + extent of B
        ext = (va.max(0) - va.min(0)) + tau + (vb.max(0) - vb.min(0))
        assert (coords <= ext * (1 + 1e-12) + 1e-9).all()
        bound = tau + da + db
        assert coords.max() <= bound * (1 + 1e-12) + 1e-9
        worst = max(worst, coords.max() / bound)
        checked += int(close.sum())
    assert checked > 1000
    # the bound is not loose by orders of magnitude on these shapes
    assert worst > 0.3
