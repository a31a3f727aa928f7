"""Replicas-only multi-GPU path of bench.py: each rank runs its own pairs and
the job's rate is every rank's pairs over the slowest rank's time. Checked
with two gloo ranks on the CPU (the arithmetic and the collective, not a
GPU)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    from datetime import timedelta

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_s = [2.0, 3.0][rank]  # rank 1 is the slow one
        t = bench.max_over_ranks(local_s, dist, "cpu")
        q.put((rank, t, bench.whole_job_rate(16, 3, world, t)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in ps)
    for rank, t, rate in res:
        assert t == 3.0
        assert rate == pytest.approx(16 * 3 * 2 / 3.0)


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(1.5, None, "cpu") == 1.5
