"""Host-side logic for running refinements on several GPUs.

A single refinement is one domain whose rounds resolve conflicts globally
(GPU_Refine/refine.cu:6830-7024), so it is not split across GPUs: each rank
refines its own input ("replicas").  Independent domains (batched
refinement) are distributed over ranks by a longest-processing-time greedy
assignment on an estimated cost, with no collective on the data path; the only
collectives are the timing reductions below.
"""
from __future__ import annotations

import heapq


def reduce_step(local_ms: float, local_triangles: float, group=None, device=None):
    """Job-wide (max time over ranks, sum of output triangles over ranks)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    n = torch.tensor([float(local_triangles)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(n.item())


def domain_cost(npoints: int, theta: float) -> float:
    """Relative work of refining one domain: output size grows with the input
    and with the angle bound (more Steiner points for larger theta)."""
    return float(npoints) * (1.0 + 0.05 * max(theta - 15.0, 0.0))


def partition_domains(costs, world: int):
    """Longest-processing-time greedy: returns one list of domain ids per rank
    (each list in ascending id order) and the per-rank total cost."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    loads = [0.0] * world
    for r in range(world):
        parts[r].sort()
        loads[r] = sum(costs[i] for i in parts[r])
    return parts, loads


def refine_batch_sharded(cdts, thetas=20.0, group=None, engine=None, gather=True, **kw):
    """Batched refinement of independent domains over the ranks of a process
    group, one GPU per rank.

    Every rank receives the same list of domains.  partition_domains assigns
    them to ranks by estimated cost (domain_cost: points and theta); each rank
    refines its share with one call of `engine` (default: the persistent batch
    engine, refine.refine_batch_persistent, on the GPU of this rank's
    LOCAL_RANK) and no data moves between GPUs.  With gather=True the results
    are collected on rank 0 by host copies (gather_object) and returned there
    in input order, as (list of CDT, list of stats dicts, report); the other
    ranks return (None, None, report).  With gather=False every rank returns
    only its own share: (its domain ids, its results, its stats, report).

    report: {"rank_ms": this rank's wall time of its engine call, "max_ms": the
    slowest rank's (the job's time), "domains": per-rank domain counts,
    "loads": per-rank estimated costs}.
    """
    import os
    import time

    import torch.distributed as dist

    n = len(cdts)
    th = [float(thetas)] * n if isinstance(thetas, (int, float)) else [float(t) for t in thetas]
    if len(th) != n:
        raise ValueError("one theta per domain")
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    costs = [domain_cost(c.numberofpoints, t) for c, t in zip(cdts, th)]
    parts, loads = partition_domains(costs, world)
    mine = parts[rank]
    if engine is None:
        from . import refine
        kw.setdefault("device", int(os.environ.get("LOCAL_RANK", 0)))

        def engine(doms, ths, **k):
            return refine.refine_batch_persistent(doms, ths, **k)
    t0 = time.perf_counter()
    res, stats = engine([cdts[i] for i in mine], [th[i] for i in mine], **kw) if mine else ([], [])
    rank_ms = (time.perf_counter() - t0) * 1e3
    max_ms, _ = reduce_step(rank_ms, 0.0, group=group, device=_reduce_device(group))
    report = {"rank_ms": rank_ms, "max_ms": max_ms, "domains": [len(p) for p in parts], "loads": loads}
    if not gather:
        return mine, res, stats, report
    share = (mine, list(res), list(stats))
    if on and world > 1:
        got = [None] * world if rank == 0 else None
        dist.gather_object(share, got, dst=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    else:
        got = [share]
    if rank != 0:
        return None, None, report
    out, out_stats = [None] * n, [None] * n
    for ids, r, s in got:
        for i, a, b in zip(ids, r, s):
            out[i], out_stats[i] = a, b
    return out, out_stats, report


def _reduce_device(group):
    """Device of the reduction tensors: the current CUDA device under NCCL,
    the host otherwise."""
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return None
