"""Multi-GPU layout of the electron step: one process per GPU over torch.distributed.

* Swarm instances (E/N points, gases, replicas) are independent: they are dealt to ranks
  by predicted work (electrons x steps, longest first; served requests online in arrival
  order) and need no collective on the data path; results are gathered on the host.
* The streamer step shards one particle population across ranks on a shared mesh.  The
  only coupling is the deposit: each rank deposits its shard into its own int64 charge
  grid and the grids are summed with an all-reduce, which is exact and independent of
  the reduction order (int64 fixed point), so the result equals a one-GPU deposit of the
  whole population.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous shard [lo, hi) of n items for `rank` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def balance_instances(work: Sequence[float], world: int) -> list[list[int]]:
    """Deal instances to ranks, longest first, each to the least-loaded rank (ties to the
    lower rank).  Deterministic: every rank computes the same assignment."""
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    for lst in out:
        lst.sort()
    return out


def my_instances(work: Sequence[float], rank: int, world: int) -> list[int]:
    """The instances rank `rank` steps (balance_instances; one rank gets them all)."""
    if world <= 1:
        return list(range(len(work)))
    return balance_instances(work, world)[rank]


def shard_requests(requests, rank: int, world: int) -> list:
    """Online dealing of served requests (arrival order): each request goes to the rank with
    the least predicted work so far (its electron count), ties to the lower rank.  Every
    rank computes the same assignment from the same arrival list, so no collective is
    needed to route a request."""
    if world <= 1:
        return list(requests)
    load = [0.0] * world
    mine = []
    for r in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        k = min(range(world), key=lambda j: (load[j], j))
        load[k] += float(r.n)
        if k == rank:
            mine.append(r)
    return mine


def gather_by_index(local: dict, n: int, group=None) -> list:
    """Every rank's {instance index: result} merged into one list of n results, on every
    rank (all_gather_object; results must be picklable)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        parts = [local]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, local, group=group)
    out = [None] * n
    for part in parts:
        for i, v in part.items():
            if out[i] is not None:
                raise ValueError(f"instance {i} was stepped by two ranks")
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"instances {missing[:8]} were stepped by no rank")
    return out


def allreduce_int64_(tensor, group=None):
    """Sum an int64 tensor over ranks in place (exact for fixed-point charges)."""
    import torch
    import torch.distributed as dist
    if tensor.dtype != torch.int64:
        raise TypeError("charge grids are int64 fixed point")
    dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def allreduce_slab_int64_(tensor, plane: int, group=None):
    """Sum an int64 charge grid over ranks in place, moving only the z-planes that hold
    charge on some rank: each rank finds its nonzero plane range, one small all-reduce gives
    the union, and the sum runs over that contiguous slab (planes outside it are zero on every
    rank).  A cloud that covers a tenth of the mesh's height moves a tenth of the bytes; the
    result is the full all-reduce's, bit for bit.  Returns the slab's plane range."""
    import torch
    import torch.distributed as dist
    if tensor.dtype != torch.int64:
        raise TypeError("charge grids are int64 fixed point")
    planes = tensor.numel() // plane
    rows = tensor.view(planes, plane).ne(0).any(dim=1)
    nz = torch.nonzero(rows).flatten()
    lo = int(nz[0]) if nz.numel() else planes
    hi = int(nz[-1]) + 1 if nz.numel() else 0
    rng = torch.tensor([-lo, hi], dtype=torch.int64, device=tensor.device)
    dist.all_reduce(rng, op=dist.ReduceOp.MAX, group=group)
    lo, hi = int(-rng[0]), int(rng[1])
    if hi > lo:
        dist.all_reduce(tensor[lo * plane:hi * plane], op=dist.ReduceOp.SUM, group=group)
    return lo, hi


def allreduce_charge(grid, which: int, group=None):
    """All-reduce a grid's device charge array in place (the NCCL int64 sum of the shards)."""
    import torch
    t = torch.as_tensor(grid.charge_array(which), device=f"cuda:{grid.ctx.device}")
    return allreduce_int64_(t, group)
