"""The multi-GPU path of bench.py is independent replicas (one mesh per
rank, no data-path collective); its only collective is the max over ranks
of the timed region.  Checked with two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], dist, "cpu")
        v = bench.replica_throughput(world, 1000, 10, t)
        Path(out_dir, f"r{rank}.txt").write_text(f"{t} {v}")
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    world, times = 2, [10.0, 12.5]
    mp.start_processes(_rank, args=(world, _free_port(), times, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        t, v = map(float, Path(tmp_path, f"r{r}.txt").read_text().split())
        assert t == 12.5
        assert v == pytest.approx(2 * 1000 * 10 / 0.0125 / 1e6)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.replica_throughput(1, 2_000_000, 5, 100.0) == pytest.approx(100.0)
