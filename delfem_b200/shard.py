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


def timed_sharded(work, solve_local, device="cpu", group=None):
    """Each rank solves its share of the instances and times it; the time of
    the job is the maximum over ranks.

    solve_local(indices) -> (seconds, results): solves the instances with the
    given indices (this rank's share, ascending) and returns its time and one
    picklable result per instance.  device: where the max-reduction tensor
    lives ("cpu" for gloo, "cuda:<n>" for NCCL).  Every rank takes the same
    collective steps (an all-reduce of the time, a gather of the results).
    Returns, on rank 0, {"seconds": max over ranks, "per_rank_instances": [...],
    "per_rank_seconds": [...], "results": [per instance, original order]}
    (None on the other ranks)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    parts = partition(work, world)
    mine = parts[rank]
    secs, local = solve_local(mine) if mine else (0.0, [])
    if len(local) != len(mine):
        raise RuntimeError("solve_local returned a wrong number of results")
    t = torch.tensor([float(secs)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    payload = (float(secs), list(zip(mine, local)))
    if world == 1:
        gathered = [payload]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(work)
    for _, part in gathered:
        for k, res in part:
            out[k] = res
    return {"seconds": float(t.item()), "per_rank_instances": [len(p) for p in parts],
            "per_rank_seconds": [g[0] for g in gathered], "results": out}
