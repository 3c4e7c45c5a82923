"""The multi-rank side of bench.py on CPU: world size 2 over gloo (the GPU run
uses NCCL with the same calls).  Every rank takes part in the same reduction;
the time is the maximum over the ranks and the throughput counts the
particles of all ranks (replicas, weak scaling)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, ms_per_rank, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms, value = bench.replica_throughput(ms_per_rank[rank], 1000, 10, dist, "cpu")
        out.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ms_per_rank = [40.0, 50.0]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ms_per_rank, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in res:
        assert ms == 50.0  # the slowest rank
        assert value == pytest.approx(1000 * 2 * 10 / 0.050)


def test_replica_throughput_one_rank():
    import bench
    ms, value = bench.replica_throughput(20.0, 500, 4)
    assert ms == 20.0 and value == pytest.approx(500 * 4 / 0.020)
