"""The multi-GPU form is replicas only (a pair does not shard): N ranks each
compute their own workload and the job's time is the slowest rank's.  This
checks bench.py's aggregation over a world-size-2 gloo process group on CPU:
both ranks see the maximum time and the whole-job rate (all ranks' units over
that time)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, results):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        t, rate = bench.replica_rate(1.0 + rank, 10.0, world, "cpu")
        results[rank] = (t, rate)
    finally:
        dist.destroy_process_group()


def test_replica_rate_max_over_ranks():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert dict(results) == {0: (2.0, 10.0), 1: (2.0, 10.0)}


def test_replica_rate_single_rank():
    import bench
    assert bench.replica_rate(0.5, 10.0, 1) == (0.5, 20.0)


def test_profiled_traffic_belongs_to_the_captured_schedule():
    """The DRAM traffic bench.py reports comes from an ncu capture of the same
    aggregation kernel: it is keyed by workload and schedule, and a schedule
    without a capture reports none."""
    import bench
    assert bench.profiled_traffic("1920x1080_d128_sad_8path", 4) == 6.42
    assert bench.profiled_traffic("1920x1080_d128_sad_8path", 6) == 13.16
    assert bench.profiled_traffic("1920x1080_d128_census_8path", 6) == 13.15
    assert bench.profiled_traffic("1920x1080_d128_sad_8path", 1) is None
    assert bench.profiled_traffic("640x480_d64_census_4path", 4) is None
