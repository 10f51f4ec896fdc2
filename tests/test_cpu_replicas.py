"""The multi-GPU path of bench.py: independent replicas (the hot path does
not shard), whose job time is the slowest rank's, all-reduced with MAX; run
here as two gloo ranks on the CPU (the GPU run uses NCCL)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [1.5, 2.5][rank]
        m = bench.max_over_ranks(ms, "cpu")
        out.put((rank, m, bench.replica_throughput(world, 1000, 10, m)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in res:
        assert m == 2.5, (rank, m)
        assert v == pytest.approx(2 * 1000 * 10 / 0.0025), (rank, v)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, "cpu") == 3.0
    assert bench.replica_throughput(1, 100, 4, 2.0) == pytest.approx(100 * 4 / 0.002)
