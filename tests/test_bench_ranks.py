"""The replica path of bench.py on CPU: two gloo ranks reduce their step
times to the slowest rank's, and the whole-job rate counts every replica."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    import bench
    ms = [2.5, 4.0][rank]
    out[rank] = bench.max_over_ranks(ms, 2, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(port, out), nprocs=2, start_method="spawn")
        assert out[0] == out[1] == 4.0


def test_replica_rate_counts_every_rank():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.replica_rate(917148808, 0.4, 1) == pytest.approx(2292.87, rel=1e-4)
    assert bench.replica_rate(917148808, 0.4, 8) == pytest.approx(8 * 2292.87, rel=1e-4)
    assert bench.max_over_ranks(3.0, 1, "cpu") == 3.0
