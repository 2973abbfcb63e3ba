"""Sharding a batch of independent systems over ranks (one process per GPU).

Instances never exchange data, so a multi-GPU batched solve is weak scaling
with no collective on the data path: every rank solves its own share of the
instances as one block-diagonal batch (delfem_b200.lib.Batch) and the only
communication is a host-side gather of the per-instance results to rank 0 at
the end.  Instances are assigned by a greedy balance of their work estimate
(largest first, each to the least-loaded rank; ties to the lower rank), which
every rank computes identically from the sizes alone.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(work, world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of instances to `world` ranks.

    work: per-instance work estimate (e.g. (n+1)^2 unknowns, or unknowns x
    expected iterations).  Returns, per rank, its instance indices ascending."""
    work = np.asarray(work, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(work.size), key=lambda k: (-work[k], k))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(work[k]), r))
    return [sorted(p) for p in parts]


def loads(work, parts) -> np.ndarray:
    work = np.asarray(work, dtype=np.float64)
    return np.array([work[p].sum() if p else 0.0 for p in parts])


def solve_sharded(instances, work, solve_local, group=None):
    """Solve `instances` (any per-instance descriptions) over the ranks of the
    default torch.distributed group (or `group`).

    solve_local(list_of_instances) -> list of per-instance results (any
    picklable objects, e.g. (x, iters, status)) runs on this rank's share.
    Returns, on rank 0, the results of all instances in their original order
    (None on the other ranks).  Every rank takes the same collective steps."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    parts = partition(work, world)
    mine = parts[rank]
    local = solve_local([instances[k] for k in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("solve_local returned a wrong number of results")
    payload = list(zip(mine, local))
    if world == 1:
        gathered = [payload]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(instances)
    for part in gathered:
        for k, res in part:
            out[k] = res
    return out
