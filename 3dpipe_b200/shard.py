"""Splitting a join over N ranks (one process per GPU).

The join's query objects are independent given tile 2: each query object's
candidates, filter and LOD refine read only its own triangles and tile 2 (the
reference's per-object candidate lists, src/join/KNNJoin.cpp:552-600, never
mix query objects; the reference itself runs on one GPU,
src/geometry/cuda_common.cu:20).  So N ranks split the query objects into
contiguous ranges of about equal estimated work (tdp_raw_partition: the voxel
pairs of each object's candidates), each rank joins its range against the
whole tile 2 -- with the range on the full tile (tdp_join_params.query_begin /
query_end, ids stay global; the way a self-join is split) or with a tile of
just its objects (local ids, mapped back with to_global) -- and no collective
touches the data path.  Only the results cross ranks at the end
(gather_results), plus whatever the caller reports (step times).
"""
from __future__ import annotations

import numpy as np


def partition(raw1, raw2=None, n_shards: int = 2, knn: int = 0, within: float = 0.0, intersect: bool = False):
    """Contiguous query ranges of about equal estimated work: bounds[n_shards + 1]
    (shard s is [bounds[s], bounds[s + 1])) and each shard's work estimate.
    raw2 None is a self-join of raw1.  Deterministic: every rank computes the
    same split from the same tiles."""
    from . import tdp
    return tdp.partition_queries(raw1, raw2, n_shards, knn=knn, within=within, intersect=intersect)


def shard_range(bounds, rank: int) -> tuple[int, int]:
    """The query range [begin, end) of `rank`."""
    if not (0 <= rank < len(bounds) - 1):
        raise ValueError("rank must be in [0, n_shards)")
    return int(bounds[rank]), int(bounds[rank + 1])


def gen_shard_tiles(begin: int, end: int, n_vessels: int, nuclei_per_vessel: int, seed: int, **kw):
    """(tile of the generated nuclei [begin, end) -- their placement as in the
    full tile, local ids 0..end-begin -- and the full vessel tile)."""
    from . import tdp
    return tdp.gen_tiles(n_vessels, nuclei_per_vessel, seed=seed, nuclei_begin=begin, nuclei_end=end, **kw)


def to_global(q_local: np.ndarray, first: int) -> np.ndarray:
    """Map a shard tile's local query ids to global ones."""
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


def gather_results(q, t, d, dst: int | None = 0):
    """Collect every rank's (global qid, rid, dist) through torch.distributed
    (any backend: the parts travel as pickled host arrays) and merge them.
    Returns the merged triple on rank dst (on every rank when dst is None),
    None on the others.  Every rank must call it."""
    import torch.distributed as dist
    part = (np.asarray(q, np.int64), np.asarray(t, np.int64), np.asarray(d, np.float64))
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return merge_results([part])
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, part)
    if dst is None or dist.get_rank() == dst:
        return merge_results(parts)
    return None
