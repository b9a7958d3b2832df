"""The multi-rank timing of bench.py (one process per GPU, time = max over
ranks) on two gloo ranks: every rank gets the slowest rank's time, and the
reference arm runs on rank 0 only."""
import os
import socket

import pytest


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        bench.barrier(world)
        got = bench.max_over_ranks(10.0 + rank * 2.5, world)

        class A:  # the reference arm returns at once on ranks other than 0
            steps, warmup = 1, 0
        ran = None
        if rank == 1:
            ran = bench.run_reference(A()) is None
        q.put((rank, got, ran))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1] == res[1][1] == 12.5
    assert res[1][2] is True
