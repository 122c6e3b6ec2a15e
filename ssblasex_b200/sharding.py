"""Batch sharding across GPUs (one process per GPU).

The instances of a batched GEMM are independent (the reference's launcher strides independent
(batch, m-block, n-block) tasks over thread teams with no cross-task reduction,
src/include/Launcher/launcher.hpp:219-230), so several GPUs split the batch into contiguous
instance ranges and each computes its own range on its own GPU. There is no collective on the
data path; a collective is used only to gather results when the caller asks for them on one rank.
"""
from __future__ import annotations


def shard_range(batch: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of the instances owned by `rank`; ranges are contiguous, disjoint, cover
    the batch, and differ in size by at most one instance."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(max(batch, 0), world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def shard_problem(p, world: int, rank: int):
    """The sub-problem (a workloads.Problem over this rank's instances) -- views, no copies."""
    import dataclasses
    s, e = shard_range(p.batch, world, rank)
    return dataclasses.replace(p, batch=e - s, A=p.A[s:e], B=p.B[s:e], C=p.C[s:e]), (s, e)


def run_sharded(p, compute, group=None, gather: bool = False):
    """Runs `compute(sub_problem) -> C_sub` on this rank's shard. With gather=True the full C is
    assembled on every rank (all_gather of the per-rank results, ordered by rank)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sub, (s, e) = shard_problem(p, world, rank)
    C_sub = compute(sub) if sub.batch > 0 else p.C[s:e].copy()
    if not gather or world == 1:
        return C_sub, (s, e)
    parts = [None] * world
    dist.all_gather_object(parts, (s, e, C_sub), group=group)
    import numpy as np
    C = p.C.copy()
    for (a, b, c) in parts:
        C[a:b] = c
    return C, (0, p.batch)
