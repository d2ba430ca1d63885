"""A cap on the within join's LODs before the last, replayed on the
reference's rules (CPU, the reference's own MeshDist).

At Hausdorff level 2 a voxel pair's bounds are running minima over the LODs,
and a pair's minmax after an LOD is at most the smallest upper bound of the
voxel pairs that LOD refines.  So a voxel pair whose lower bound comes out
above C = max(tau, that upper bound) (widened a little) can keep its previous
bounds: where they are at most C they are the exact running minima, and above
C no rule reads them (the eviction drops the voxel pair, the drop rule needs
only "above tau").  The result set must be the same with and without the
cap on every seeded within case; the counts show how much of the refine the
cap would spare at those LODs.
"""
import numpy as np
import pytest

from join_cases import CASES, tiles
from oracle_bind import ref_join, ref_join_capped, reference

WITHIN_L2 = [n for n, c in CASES.items() if c[3] == "within" and c[8] == 2]


@pytest.mark.skipif(reference() is None, reason="the reference's CPU code was not built")
@pytest.mark.parametrize("name", WITHIN_L2)
def test_capped_lods_keep_the_result_set(name):
    nv, npv, seed, _query, _knn, tau, self_join, lods, _level = CASES[name]
    nb, vb = tiles(nv, npv, seed)
    t2 = None if self_join else vb
    q0, t0, _ = ref_join(nb, t2, self_join, False, tau=tau, lods=lods, level=2)
    q1, t1, capped = ref_join_capped(nb, t2, self_join, tau, 1e-4, lods=lods)
    assert np.array_equal(q0, q1) and np.array_equal(t0, t1)
    assert (capped >= 0).all()


def test_caps_spare_part_of_the_refine():
    if reference() is None:
        pytest.skip("the reference's CPU code was not built")
    spared = 0.0
    for name in WITHIN_L2:
        nv, npv, seed, _query, _knn, tau, self_join, lods, _level = CASES[name]
        nb, vb = tiles(nv, npv, seed)
        _, _, capped = ref_join_capped(nb, None if self_join else vb, self_join, tau, 1e-4, lods=lods)
        spared += capped[1]
    assert spared > 0
