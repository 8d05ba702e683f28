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
