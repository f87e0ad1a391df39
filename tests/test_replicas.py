"""Multi-GPU is replicas only (one independent SpMV per rank, no exchange step).  The rank
plumbing bench.py uses for N > 1 -- barrier, time as the max over ranks, whole-job value
as the sum of the replicas -- on two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        local_ms = 1.0 + rank                       # rank 1 is the slower replica
        ms = bench.max_over_ranks(world, local_ms)
        B = 1_000_000
        value = world * B * 1e-9 / (ms * 1e-3)      # whole-job GB/s of N replicas
        bench.barrier(world)
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_replicas_barrier_and_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [2.0, 2.0]          # both ranks report the slowest replica's time
    assert res[0][2] == pytest.approx(2 * 1e6 * 1e-9 / 2e-3)
