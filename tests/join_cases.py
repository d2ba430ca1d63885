"""Seeded join workloads shared by the CPU and GPU join tests (small shapes of
the benchmark configurations: nuclei around vessels on a 1000-unit grid)."""
from __future__ import annotations

import functools
import importlib

import numpy as np


@functools.lru_cache(maxsize=None)
def tiles(n_vessels: int, nuclei_per_vessel: int, seed: int):
    pkg = importlib.import_module("3dpipe_b200")
    nb, vb = pkg.tdp.gen_tiles(n_vessels, nuclei_per_vessel, seed=seed)
    return nb, vb


# name -> (n_vessels, nuclei_per_vessel, seed, query, knn, tau, self_join, lods, level)
CASES = {
    "knn3_nuc_ves": (6, 12, 101, "nn", 3, 0.0, False, None, 2),
    "knn1_nuc_ves": (8, 10, 102, "nn", 1, 0.0, False, None, 2),
    "within150": (6, 12, 103, "within", 0, 150.0, False, None, 2),
    "within400": (8, 10, 104, "within", 0, 400.0, False, None, 2),
    "knn5_self": (4, 16, 105, "nn", 5, 0.0, True, None, 2),
    "within60_self": (4, 16, 106, "within", 0, 60.0, True, None, 2),
    "knn3_lod100_only": (6, 12, 101, "nn", 3, 0.0, False, [100], 2),
    "within150_lod20_100": (6, 12, 103, "within", 0, 150.0, False, [20, 100], 2),
    "knn3_level0": (6, 12, 101, "nn", 3, 0.0, False, None, 0),
    "within150_level1": (6, 12, 103, "within", 0, 150.0, False, None, 1),
}


def exact_truth(nb, vb, self_join, query, knn, tau):
    """FP64 exact result set and the smallest decision margin (near-tie check)."""
    from oracle_bind import join_exact
    q, t, d, inn = join_exact(nb, None if self_join else vb, self_join, query == "nn", knn=knn, tau=tau)
    res = set(zip(q[inn].tolist(), t[inn].tolist()))
    if query == "nn":
        margin = np.inf
        for qi in np.unique(q):
            m = q == qi
            ds = np.sort(d[m])
            if len(ds) > knn:
                margin = min(margin, ds[knn] - ds[knn - 1])
    else:
        margin = float(np.abs(d - tau).min()) if len(d) else np.inf
    return res, margin
