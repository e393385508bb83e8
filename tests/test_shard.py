"""Placement of whole clouds on the GPUs of a node (host logic, CPU): the
batched workload's clouds spread over 2-8 ranks, balanced by work within a
memory budget, and every rank computing the same placement on its own."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from mlodsurfaces_b200 import shard

ROOT = Path(__file__).resolve().parents[1]


def test_largest_first_balances_and_is_deterministic():
    rng = np.random.default_rng(3)
    work = np.exp(rng.uniform(np.log(1e4), np.log(4e6), 64))
    nbytes = [shard.cloud_bytes(int(w), int(w)) for w in work]
    for n in (1, 2, 3, 4, 8):
        a = shard.assign_clouds(work, nbytes, n)
        assert a == shard.assign_clouds(list(work), list(nbytes), n)
        assert sorted(set(a)) == list(range(n))
        load = np.bincount(a, weights=work, minlength=n)
        assert load.max() <= work.sum() / n + work.max() + 1e-6
        assert np.isclose(load.sum(), work.sum())


def test_memory_budget_is_respected_and_impossible_placements_fail():
    work = [10, 9, 8, 7, 1]
    nbytes = [100, 100, 100, 100, 100]
    a = shard.assign_clouds(work, nbytes, 3, capacity=200)
    used = np.bincount(a, weights=nbytes, minlength=3)
    assert used.max() <= 200
    with pytest.raises(ValueError):
        shard.assign_clouds(work, nbytes, 2, capacity=200)  # 500 bytes do not fit in 2 x 200
    with pytest.raises(ValueError):
        shard.assign_clouds([1.0], [1000], 4, capacity=999)
    with pytest.raises(ValueError):
        shard.assign_clouds([1.0], [1, 2], 1)


def test_bench_batch_placement_covers_every_cloud():
    sys.path.insert(0, str(ROOT))
    import bench

    specs = bench.batch_cloud_specs(64)
    again = bench.batch_cloud_specs(64)  # seeded: a fixed workload
    assert [(s["n"], s["kind"], s["depth"]) for s in specs] == [(s["n"], s["kind"], s["depth"]) for s in again]
    assert 3e7 < sum(s["n"] for s in specs) < 6e7
    work = np.array([s["n"] for s in specs], float)
    for world in (2, 4, 8):
        place = bench.batch_placement(specs, world, 1)
        assert len(place) == 64 and set(place) == set(range(world))
        load = np.bincount(place, weights=work, minlength=world)
        assert load.max() <= work.sum() / world + work.max()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        place = bench.batch_placement(bench.batch_cloud_specs(64), world, 1)
        got = [None] * world
        dist.all_gather_object(got, place)
        np.save(Path(out_dir) / f"rank{rank}.npy", np.array(got))
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_the_placement_without_exchanging_it(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g0 = np.load(tmp_path / "rank0.npy")
    g1 = np.load(tmp_path / "rank1.npy")
    assert np.array_equal(g0, g1) and np.array_equal(g0[0], g0[1])
