"""Multi-process plumbing: one process per GPU over torch.distributed, no collective on the data path.

* One LP does not shard without an all-gather of x_bar and one of y per iteration, so single
  LPs run as independent replicas (one LP per rank); a timing is reduced as the maximum over
  ranks.
* A batch of independent LPs shards naturally: the instances are partitioned across ranks by
  their nonzero counts (longest-processing-time greedy), each rank solves its shard with one
  vajra_pdhg_solve_batch call, and the per-instance summaries are gathered once at the end.

The collectives here are host-side bookkeeping (a handful of scalars and small dicts); they run
on any backend (NCCL on a multi-GPU node, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq


def partition_by_nnz(nnz, world: int) -> list:
    """Indices of `nnz` split into `world` shards of near-equal total (LPT greedy).

    Deterministic: ties break on the lower index / rank, and every shard lists its indices
    in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(nnz)), key=lambda i: (-int(nnz[i]), i))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(nnz[i]), r))
    return [sorted(s) for s in shards]


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The maximum of a per-rank scalar over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj, dist=None) -> list:
    """Every rank's `obj`, in rank order (a one-element list without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def summarize(result: dict) -> dict:
    """The scalar part of one solve_batch result (what crosses ranks; vectors stay local)."""
    keys = ("status", "status_name", "iterations", "objective_value", "rel_kkt", "device_time_sec")
    return {k: result[k] for k in keys if k in result}


def solve_batch_sharded(lps, rank: int, world: int, dist=None, solve_batch=None, **opts):
    """Solve this rank's shard of `lps`; gather every rank's per-instance summaries.

    Returns (shard indices, local full results, summaries of all instances in input order).
    `solve_batch` defaults to vajra_pdhg.solve_batch (a stand-in can be passed for tests)."""
    if solve_batch is None:
        from . import solve_batch as solve_batch_impl
        solve_batch = solve_batch_impl
    shards = partition_by_nnz([lp.nnz for lp in lps], world)
    mine = shards[rank]
    local = solve_batch([lps[i] for i in mine], **opts) if mine else []
    gathered = gather_objects([(i, summarize(r)) for i, r in zip(mine, local)], dist)
    summaries = [None] * len(lps)
    for part in gathered:
        for i, s in part:
            summaries[i] = s
    return mine, local, summaries
