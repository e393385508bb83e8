"""The multi-rank benchmark path on CPU: two gloo ranks, each with its own
replica of the cloud and its own queries, reduce their timings to the max
over ranks; the job throughput counts every rank's queries."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pts, nrm, q, diag, k = bench.workload(3000, rank)
        # rank-dependent step times: the job time is the slowest rank's
        times = bench.max_over_ranks([10.0 + rank, 5.0 * (world - rank)], world, torch.device("cpu"))
        np.savez(Path(out_dir) / f"rank{rank}.npz", pts=pts, q=q, times=np.array(times))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replicate_the_cloud_and_take_the_max(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert np.array_equal(r0["pts"], r1["pts"])  # every rank builds the same tree
    assert not np.array_equal(r0["q"], r1["q"])  # each rank projects its own queries
    assert list(r0["times"]) == [11.0, 10.0] and list(r1["times"]) == [11.0, 10.0]


def test_job_throughput_counts_all_ranks():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.job_throughput(1, 1000, 10, 1000.0) == pytest.approx(10000.0)
    assert bench.job_throughput(4, 1000, 10, 1000.0) == pytest.approx(40000.0)
