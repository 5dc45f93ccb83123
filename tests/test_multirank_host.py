"""The N > 1 path of bench.py on CPU: two gloo ranks (replicas only, no data
exchange) agree on the slowest rank's timings, and the whole-job throughput
counts every rank's frames.  The reference arm runs on rank 0 alone."""

import os
import socket
import sys
import types

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        times = bench.max_over_ranks([100.0 * (rank + 1), 7.0 - rank], dist, "cpu")
        reference = bench.run_reference(types.SimpleNamespace(steps=1, warmup=0), rank) if rank != 0 else None
        out.put((rank, times, reference))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict((r, (t, ref)) for r, t, ref in (out.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0][0] == results[1][0] == [200.0, 7.0]
    assert results[1][1] is None  # only rank 0 runs the reference arm


def test_whole_job_throughput_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_throughput(1000, 1, 1000.0) == pytest.approx(1000.0)
    assert bench.replica_throughput(1000, 4, 1250.0) == pytest.approx(3200.0)
