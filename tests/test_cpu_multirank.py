"""The multi-rank path of bench.py on CPU: two gloo ranks agree on the slowest rank's time
(max over ranks), and the job value counts every rank's grid (replicas, no data-path
collective)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 10.0 + 5.0 * rank              # rank 1 is the slow one
        got = bench.max_over_ranks(local, dist, "cpu")
        with open(os.path.join(out_dir, "r%d" % rank), "w") as f:
            f.write(repr(got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert [float(open(os.path.join(tmp_path, "r%d" % r)).read()) for r in range(2)] == [15.0, 15.0]


def test_job_value_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.job_value(1, 1_000_000, 2.0)
    assert one == pytest.approx(500.0)
    assert bench.job_value(4, 1_000_000, 2.0) == pytest.approx(4 * one)
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
