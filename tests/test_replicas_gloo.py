"""Replica (one process per GPU) plumbing of bench.py on CPU: two gloo ranks
take the same collective steps and agree on the slowest rank's time, which
is what `value` divides the whole job's bytes by."""
import datetime
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(ws)
        ms = 10.0 + 5.0 * rank  # the second rank is the slow one
        q.put((rank, bench.max_over_ranks(ms, ws)))
        bench.barrier(ws)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(ws))
    assert got == {0: 15.0, 1: 15.0}


def _rank_tail(rank, ws, port, q):
    """The tail of bench.run_ours: the last collective, then rank 0 alone works
    on (its rates and reports) while the other ranks leave the group."""
    import time

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=5))
    try:
        bench.barrier(ws)
        e2e_ms = bench.max_over_ranks(3.0 + rank, ws)
        if rank == 0:
            time.sleep(8.0)  # longer than the group's timeout
        q.put((rank, e2e_ms))
    finally:
        dist.destroy_process_group()


def test_rank0_work_after_the_last_collective_outlasts_the_timeout():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_tail, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(ws))
    assert got == {0: 4.0, 1: 4.0}
