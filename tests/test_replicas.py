"""The multi-GPU path is replicas only (independent solves, no collective on
the data path): what crosses ranks is the timing.  Two gloo ranks on the CPU
check the max-over-ranks reduction and the whole-job figure bench.py uses."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    got = bench.max_over_ranks(torch, dist, ms, "cpu")
    val = bench.replicas_value(1e9, world, got)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, val))


def test_two_gloo_ranks_reduce_to_the_slowest():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, val in out:
        assert got == 150.0
        assert val == pytest.approx(2 * 1e9 / 0.150 / 1e9)
