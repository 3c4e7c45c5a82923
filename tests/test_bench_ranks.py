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


def test_reference_cpu_baseline_runs_the_reference(tmp_path, monkeypatch):
    """The CPU baseline and the reference arm run the reference's own particle
    path (compiled from its headers into oracle/_ref by oracle/build_ref.sh) on
    the bench's workload, a 2x2 grid of forked ranks here (the 64^3 uniform
    workload), with per-step times; without that build the bench falls back
    to the port."""
    import bench
    if not os.access(bench.REF_DRIVER, os.X_OK):
        pytest.skip("oracle/_ref not built (the reference sources are absent)")
    assert bench._ref_grid(4) == (2, 2) and bench._ref_grid(3) is None
    assert bench._ref_grid(200) == (8, 8)
    monkeypatch.setenv("LF2_REF_INPUT_DIR", str(tmp_path))
    r = bench.cpu_reference_steps("c1", 4, 3, 1)
    assert r is not None
    assert r["ranks"] == 4 and r["steps"] == 3 and r["warmup"] == 1
    assert len(r["step_seconds"]) == 3 and r["particles_after"] == 64 ** 3
    cpu = bench.cpu_reference_summary("c1", r)
    assert cpu["kind"] == "reference" and cpu["cores"] == 4 and cpu["value"] > 0
    assert bench.workload_config("c3")["particles"] == 512 ** 3
