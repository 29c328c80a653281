"""The replica path of the bench (N independent copies, one process per GPU)
on CPU: two gloo ranks agree on the slowest rank's time and on the whole-job
rate, and exchange nothing else."""
from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp

from stipple_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        my_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        slow = replicas.max_over_ranks(my_ms)
        rate = replicas.job_rate(1000.0, world, slow)
        q.put((rank, slow, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slow, rate in got:
        assert slow == 150.0
        assert rate == world * 1000.0 / 0.150


def test_single_process_is_identity():
    assert replicas.max_over_ranks(12.5) == 12.5
    assert replicas.job_rate(10.0, 1, 1000.0) == 10.0
