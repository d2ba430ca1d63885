"""The N-rank join path on CPU: two gloo ranks each join their own vessel
block's nuclei (generated with the rank's nuclei range) against the full
vessel tile with the FP64 oracle; the gathered union, with local query ids
mapped back to global ones, must equal the single-process join, and the
reported step time is the max over ranks."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CASE = dict(n_vessels=4, nuclei_per_vessel=6, seed=20260011)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, query, out_dir):
    import importlib

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg = importlib.import_module("3dpipe_b200")
        from oracle_bind import join_exact
        nb, vb, first = pkg.shard.gen_shard_tiles(rank, world, CASE["n_vessels"], CASE["nuclei_per_vessel"],
                                                  CASE["seed"])
        q, t, d, inn = join_exact(nb, vb, False, query == "nn", knn=3, tau=150.0)
        part = (pkg.shard.to_global(q[inn], first), t[inn], d[inn])
        parts = [None] * world
        dist.all_gather_object(parts, part)
        step = torch.tensor([1.0 + rank], dtype=torch.float64)
        dist.all_reduce(step, op=dist.ReduceOp.MAX)
        if rank == 0:
            gq, gt, gd = pkg.shard.merge_results(parts)
            np.savez(Path(out_dir) / f"{query}.npz", q=gq, t=gt, d=gd, step=step.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("query", ["within", "nn"])
def test_two_rank_shards_union_equals_whole_join(tmp_path, query, orc):
    import importlib

    import torch.multiprocessing as mp
    from oracle_bind import join_exact
    pkg = importlib.import_module("3dpipe_b200")
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), query, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(tmp_path / f"{query}.npz")
    nb, vb = pkg.tdp.gen_tiles(CASE["n_vessels"], CASE["nuclei_per_vessel"], seed=CASE["seed"])
    q, t, d, inn = join_exact(nb, vb, False, query == "nn", knn=3, tau=150.0)
    o = np.lexsort((t[inn], q[inn]))
    np.testing.assert_array_equal(got["q"], q[inn][o])
    np.testing.assert_array_equal(got["t"], t[inn][o])
    np.testing.assert_allclose(got["d"], d[inn][o], rtol=0, atol=0)
    assert float(got["step"][0]) == 2.0  # max over ranks
    assert len(got["q"]) > 0


def test_vessel_blocks_partition():
    import importlib
    pkg = importlib.import_module("3dpipe_b200")
    for world in (1, 2, 3, 4, 8):
        blocks = [pkg.shard.vessel_block(r, world, 1000) for r in range(world)]
        assert blocks[0][0] == 0 and blocks[-1][1] == 1000
        assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
    with pytest.raises(ValueError):
        pkg.shard.vessel_block(2, 2, 10)
