"""Multi-GPU runs of bench.py are replicas: every rank steps its own copy and
the only collectives are the barrier and the max over ranks of the timings.
That aggregation is checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms_local = 100.0 + 50.0 * rank      # rank 1 is the slow one
    ms = bench.max_over_ranks(ms_local, dist)
    dist.barrier()
    q.put((rank, ms, bench.whole_job_rate(world, 20, ms)))
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in out:
        assert ms == 150.0                       # every rank sees the max
        assert rate == pytest.approx(2 * 20 / 0.150)  # whole job: 2 replicas x 20 steps


def test_single_process_has_no_collective():
    assert bench.max_over_ranks(12.5, None) == 12.5
    assert bench.whole_job_rate(1, 10, 50.0) == pytest.approx(200.0)
