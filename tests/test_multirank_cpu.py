"""The N-rank join path on CPU: two gloo ranks each compute the query split
with the product's partitioner (tdp_raw_partition, host code, the same on
every rank), join their own query range against the whole tile 2, and gather
the results with the product's gather (shard.gather_results).  The union must
equal the single-process join.  A rank's join here is the reference's join
rules on the CPU for exactly its queries (the GPU join needs a GPU; the
single-GPU test tests/test_shard_gpu.py runs the product join per range), so
this test covers the product's split and merge, the per-query independence
that makes the split exact, and the max-over-ranks step time."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CASE = dict(n_vessels=4, nuclei_per_vessel=6, seed=20260011)
QUERIES = {"within": dict(query="within", knn=0, tau=150.0, self_join=False),
           "nn": dict(query="nn", knn=3, tau=0.0, self_join=False),
           "nn_self": dict(query="nn", knn=4, tau=0.0, self_join=True)}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case_tiles():
    import importlib
    pkg = importlib.import_module("3dpipe_b200")
    return pkg.tdp.gen_tiles(CASE["n_vessels"], CASE["nuclei_per_vessel"], seed=CASE["seed"])


def _rank_main(rank, world, port, name, out_dir):
    import importlib

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg = importlib.import_module("3dpipe_b200")
        from oracle_bind import ref_join
        c = QUERIES[name]
        nb, vb = _case_tiles()
        t2 = None if c["self_join"] else vb
        bounds, work = pkg.shard.partition(nb, t2, world, knn=c["knn"], within=c["tau"])
        every = [None] * world
        dist.all_gather_object(every, bounds.tolist())
        assert all(b == every[0] for b in every)  # the same split on every rank
        b, e = pkg.shard.shard_range(bounds, rank)
        q, t, _ = ref_join(nb, t2, c["self_join"], c["query"] == "nn", knn=c["knn"], tau=c["tau"],
                           queries=np.arange(b, e, dtype=np.int32))
        assert q.size == 0 or (q.min() >= b and q.max() < e)
        merged = pkg.shard.gather_results(q, t, np.zeros(len(q)), dst=0)
        step = torch.tensor([1.0 + rank], dtype=torch.float64)
        dist.all_reduce(step, op=dist.ReduceOp.MAX)
        if rank == 0:
            gq, gt, _ = merged
            np.savez(Path(out_dir) / f"{name}.npz", q=gq, t=gt, step=step.numpy(), bounds=bounds, work=work)
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", list(QUERIES))
def test_two_rank_shards_union_equals_whole_join(tmp_path, name, orc):
    import torch.multiprocessing as mp
    from oracle_bind import ref_join
    if not (ROOT / "oracle" / "_ref" / "libtdp_ref.so").exists():
        pytest.skip("the reference library is built from the reference sources")
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), name, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(tmp_path / f"{name}.npz")
    c = QUERIES[name]
    nb, vb = _case_tiles()
    q, t, _ = ref_join(nb, None if c["self_join"] else vb, c["self_join"], c["query"] == "nn", knn=c["knn"],
                       tau=c["tau"])
    np.testing.assert_array_equal(got["q"], q)
    np.testing.assert_array_equal(got["t"], t)
    assert float(got["step"][0]) == 2.0  # max over ranks
    assert len(got["q"]) > 0
    b = got["bounds"]
    assert b[0] == 0 and b[-1] == CASE["n_vessels"] * CASE["nuclei_per_vessel"] and (np.diff(b) >= 0).all()


@pytest.mark.parametrize("n_shards", [1, 2, 3, 5, 8, 40])
def test_partition_is_contiguous_and_balanced(pkg, n_shards):
    """Shards tile [0, n1) in order; each shard's estimated work is within one
    object's work of the even share (objects are not split)."""
    nb, vb = pkg.tdp.gen_tiles(6, 10, seed=77)
    n1 = 60
    for kw in (dict(within=200.0), dict(knn=3)):
        bounds, work = pkg.shard.partition(nb, vb, n_shards, **kw)
        assert bounds[0] == 0 and bounds[-1] == n1 and (np.diff(bounds) >= 0).all()
        one = pkg.shard.partition(nb, vb, n1, **kw)[1]  # work of every single object (n1 shards of one)
        assert np.isclose(work.sum(), one.sum())
        assert work.max() <= work.sum() / n_shards + one.max() + 1e-6
        # the same split every time
        np.testing.assert_array_equal(bounds, pkg.shard.partition(nb, vb, n_shards, **kw)[0])


def test_partition_errors(pkg):
    nb, _ = pkg.tdp.gen_tiles(2, 3, seed=5)
    with pytest.raises(pkg.TdpError):
        pkg.shard.partition(nb, None, 0, knn=1)
    with pytest.raises(pkg.TdpError):
        pkg.shard.partition(np.zeros(9, np.uint8), None, 2, knn=1)
    with pytest.raises(ValueError):
        pkg.shard.shard_range(np.array([0, 3, 6]), 2)
