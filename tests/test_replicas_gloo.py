"""The multi-GPU path of bench.py is replicas (one update does not shard):
every rank runs the same workload and the job's value is all ranks' units
over the slowest rank's time. Checked here with two gloo ranks on CPU."""
import os
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [400.0, 1000.0][rank]          # rank 1 is the slow one
        value, total_ms = bench.replica_throughput(49117, 10, local_ms, world, dist, "cpu")
        e2e = bench.max_over_ranks([7.5, 3.25][rank], dist, "cpu")
        out.put((rank, value, total_ms, e2e))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(2))
    for rank, value, total_ms, e2e in res:
        assert total_ms == 1000.0                 # the slowest rank's time
        assert value == pytest.approx(2 * 49117 * 10 / 1.0)
        assert e2e == 7.5


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    value, total_ms = bench.replica_throughput(100, 4, 200.0, 1, None, "cpu")
    assert total_ms == 200.0 and value == pytest.approx(2000.0)
