"""Sharding one proof's hot path over the GPUs of a node (one process per GPU).

The reference proves on one GPU (src/lib.rs:213-216).  The work of a proof
splits cleanly along two axes:

* commitments: every MSM of a phase is independent, so each rank commits a
  contiguous range of the phase's columns and the affine commitments (64
  bytes each) are all-gathered in column order, the only exchange the
  transcript needs (every rank then squeezes the same challenges);
* the quotient: the extended domain is E cosets of the base domain and every
  constraint of a coset reads only that coset's rows, so rank r evaluates
  cosets r, r + world, ... and the coset values of h (n field elements each)
  are all-gathered before the combine.

Everything else (grand products, evaluations, the multi-open) is small and
runs on every rank.  The collectives are torch.distributed calls: NCCL over
NVLink between GPUs; gloo serves the host-side tests.  No TMA multicast is
involved anywhere.
"""
from __future__ import annotations

import torch


def column_ranges(ncols: int, world: int) -> list:
    """Contiguous, balanced [start, stop) ranges of ncols columns, one per
    rank (the first ncols % world ranks take one more)."""
    if world < 1:
        raise ValueError("world size must be positive")
    base, extra = divmod(ncols, world)
    out, s = [], 0
    for r in range(world):
        e = s + base + (1 if r < extra else 0)
        out.append((s, e))
        s = e
    return out


def coset_ranks(cosets: int, world: int) -> list:
    """Rank r evaluates cosets r, r + world, ... of the extended domain."""
    return [list(range(r, cosets, world)) for r in range(world)]


def _dist():
    import torch.distributed as dist

    return dist


class ThreadGroup:
    """An in-process group whose ranks are threads of one process driving one
    GPU each (or sharing one): the exchanges happen on the host through a
    barrier, so no rank's kernels ever wait on another's.  It runs the sharded
    schedule's logic on a single GPU (the tests) with the same calls as a
    torch.distributed group."""

    def __init__(self, world: int):
        import threading

        self.world = world
        self.barrier = threading.Barrier(world)
        self.slots = [None] * world

    def view(self, rank: int):
        return _ThreadRank(self, rank)


class _ThreadRank:
    def __init__(self, g, rank):
        self.g, self.rank, self.world = g, rank, g.world

    def all_gather(self, obj):
        self.g.barrier.wait()
        self.g.slots[self.rank] = obj
        self.g.barrier.wait()
        out = list(self.g.slots)
        self.g.barrier.wait()
        return out


def rank_world(group) -> tuple:
    """(rank, world size) of a torch.distributed group or a ThreadGroup rank."""
    if isinstance(group, _ThreadRank):
        return group.rank, group.world
    dist = _dist()
    return dist.get_rank(group), dist.get_world_size(group)


def gather_points(local_points: list, group=None) -> list:
    """All-gather every rank's list of affine points (x, y) and return them in
    rank order, i.e. in column order when each rank holds column_ranges'
    range."""
    if isinstance(group, _ThreadRank):
        parts = group.all_gather(list(local_points))
    else:
        dist = _dist()
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, list(local_points), group=group)
    out = []
    for p in parts:
        out.extend(tuple(q) for q in p)
    return out


def gather_cosets(h: torch.Tensor, mine: list, cosets: int, group=None) -> torch.Tensor:
    """h: (cosets, n, 4) with this rank's cosets (coset_ranks) filled in;
    returns h with every coset filled, from one all-gather of equally sized
    blocks (ranks with fewer cosets pad theirs)."""
    _, world = rank_world(group)
    per = -(-cosets // world)
    n = h.shape[1]
    block = torch.zeros((per, n, 4), dtype=h.dtype, device=h.device)
    for i, j in enumerate(mine):
        block[i].copy_(h[j])
    if isinstance(group, _ThreadRank):
        torch.cuda.synchronize() if block.is_cuda else None
        parts = group.all_gather(block)
    else:
        dist = _dist()
        on_host = dist.get_backend(group) != "nccl" and h.is_cuda
        src = block.cpu() if on_host else block
        parts = [torch.empty_like(src) for _ in range(world)]
        dist.all_gather(parts, src, group=group)
    owners = coset_ranks(cosets, world)
    for r in range(world):
        for i, j in enumerate(owners[r]):
            h[j].copy_(parts[r][i])
    return h
