"""CPU test of the multi-GPU bench logic (replicas only) with world_size 2 over
gloo: the max-over-ranks reduction and the whole-job value that bench.py
reports under torchrun."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, world)
        value = bench.replica_value(1_000_000, ms_max, world)
        q.put((rank, ms_max, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms_max, value in got:
        assert ms_max == 15.0  # the max, on every rank
        assert value == pytest.approx(2 * 1_000_000 / 0.015 / 1e6)  # both ranks' elements / max time
