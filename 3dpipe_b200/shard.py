"""Sharding of a join over N ranks (one process per GPU).

The join's query objects are independent given tile 2: each query object's
candidates, filter and LOD refine read only its own triangles and the
resident tile 2 (the reference's per-object candidate lists,
src/join/KNNJoin.cpp:552-600, never mix query objects).  So N ranks split the
query tile and run whole joins with no data-path collective.  For the generated workload the
split is by vessel block: rank r generates and joins the nuclei of vessels
[v0, v1), all vessels replicated, and a query's local id maps back to the
global id by adding the block's first nucleus.  Only reporting crosses ranks
(max of the step times, sum of the pair counts, optionally a gather of the
result pairs).
"""
from __future__ import annotations

import numpy as np


def vessel_block(rank: int, world: int, n_vessels: int) -> tuple[int, int]:
    """The contiguous vessel block [v0, v1) of `rank` among `world` ranks."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    return rank * n_vessels // world, (rank + 1) * n_vessels // world


def nuclei_range(rank: int, world: int, n_vessels: int, nuclei_per_vessel: int) -> tuple[int, int]:
    """Global ids [begin, end) of the nuclei rank `rank` joins."""
    v0, v1 = vessel_block(rank, world, n_vessels)
    return v0 * nuclei_per_vessel, v1 * nuclei_per_vessel


def gen_shard_tiles(rank: int, world: int, n_vessels: int, nuclei_per_vessel: int, seed: int, **kw):
    """(nuclei tile of this rank's block, full vessel tile, first global nucleus id)."""
    from . import tdp
    b, e = nuclei_range(rank, world, n_vessels, nuclei_per_vessel)
    nb, vb = tdp.gen_tiles(n_vessels, nuclei_per_vessel, seed=seed, nuclei_begin=b, nuclei_end=e, **kw)
    return nb, vb, b


def to_global(q_local: np.ndarray, first: int) -> np.ndarray:
    """Map a shard's local query ids to global ones."""
    return np.asarray(q_local, np.int64) + int(first)


def merge_results(parts) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Union of per-rank (global qid, rid, dist) triples, sorted by (qid, rid)."""
    if not parts:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float32)
    q = np.concatenate([np.asarray(p[0], np.int64) for p in parts])
    t = np.concatenate([np.asarray(p[1], np.int64) for p in parts])
    d = np.concatenate([np.asarray(p[2], np.float64) for p in parts])
    o = np.lexsort((t, q))
    return q[o], t[o], d[o]
