"""Multi-GPU form of the benchmark: independent replicas (the residual path
does not shard), timed by the slowest rank.  The rank logic runs here as
two gloo processes on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank k "took" (k + 1) * 10 ms; every rank learns the slowest
    t = bench.max_over_ranks(10.0 * (rank + 1), dist)
    v = bench.replica_throughput(world, 500_000, 3, 200, t / 1e3)
    out.put((rank, t, v))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_whole_job_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [20.0, 20.0]
    assert got[0][2] == got[1][2] == pytest.approx(2 * 500_000 * 3 * 200 / 0.020)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_throughput(1, 10, 3, 2, 0.5) == 120.0
