"""Sharding of independent systems across ranks (one process per GPU).

Batched and served solves are independent systems: each rank takes a subset
and solves it on its own GPU; nothing crosses ranks on the data path.  The
only collectives are host-side bookkeeping over torch.distributed (gloo or
NCCL): the max of the per-rank times, and gathering summaries at rank 0.
"""
from __future__ import annotations


def assign(work, world):
    """Greedy longest-processing-time assignment of items with estimated
    work `work[i]` to `world` ranks; returns a list of index lists.  The
    result depends only on the inputs, so every rank computes the same."""
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += work[i]
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value, world):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, world):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_root(obj, world, rank):
    if world <= 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
