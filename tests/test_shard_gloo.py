"""Sharding of a proof over several GPUs (zkwasm-prover_b200/shard.py), its
host-side plumbing on two gloo ranks on the CPU: the column ranges cover every
column once and in order, the coset assignment covers every coset once, the
all-gathered commitments come back in column order, and the gathered coset
blocks land at their coset indices (uneven counts included).  The NCCL path
runs the same calls on GPUs; it is not measured on more than one GPU here."""
import importlib
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_ranges_cover_everything():
    S = importlib.import_module("zkwasm-prover_b200.shard")
    for ncols in (0, 1, 7, 121, 193):
        for world in (1, 2, 3, 8):
            r = S.column_ranges(ncols, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == ncols
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1
    for E in (2, 4, 8):
        for world in (1, 2, 3, 8):
            owned = sorted(j for js in S.coset_ranks(E, world) for j in js)
            assert owned == list(range(E))


def _worker(rank, world, port, ncols, E, n):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    S = importlib.import_module("zkwasm-prover_b200.shard")
    a, b = S.column_ranges(ncols, world)[rank]
    # a stand-in commitment of column c: (c, 1000 + c)
    got = S.gather_points([(c, 1000 + c) for c in range(a, b)])
    assert got == [(c, 1000 + c) for c in range(ncols)]
    mine = S.coset_ranks(E, world)[rank]
    h = torch.zeros((E, n, 4), dtype=torch.int64)
    for j in mine:
        h[j] = j * 10 + 1
    S.gather_cosets(h, mine, E)
    for j in range(E):
        assert (h[j] == j * 10 + 1).all()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,ncols,E", [(2, 121, 8), (3, 38, 8), (2, 3, 4)])
def test_gather_order_on_gloo(world, ncols, E):
    mp.start_processes(_worker, args=(world, _free_port(), ncols, E, 16), nprocs=world, start_method="spawn",
                       join=True)
