"""The benchmark's multi-GPU path is replicas: N ranks run independent
copies and the job's figure is every rank's work over the slowest rank's
time.  The cross-rank part runs here on CPU with two gloo ranks."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(times[rank], dist, "cpu")
        q.put((rank, slowest, bench.replica_value(3e11, world, slowest)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, times = 2, [1.25, 1.5]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, slowest, value in got:
        assert slowest == 1.5
        assert abs(value - 3e11 * 2 / 1.5 / 1e9) < 1e-9


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.5) == 2.5
    assert bench.replica_value(1e9, 1, 0.5) == 2.0
