"""The replica bookkeeping of bench.py across two ranks on the CPU (gloo):
every rank sees the slowest rank's time, and the whole-job rate counts the
points of all ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "senga-versiona_b200"))
    import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = replicas.max_over_ranks(10.0 + rank)  # rank 1 is the slower one
        rate = replicas.job_rate(1000, 5, world, t)
        out.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_on_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[0][2] == pytest.approx(1000 * 5 * 2 / 11.0)


def test_single_process_passes_values_through():
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "senga-versiona_b200"))
    import replicas

    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(10, 5, 1, 2.0) == 25.0
