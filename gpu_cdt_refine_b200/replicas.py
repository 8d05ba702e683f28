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


class ShardError(RuntimeError):
    """A rank's engine failed; raised on every rank after the collectives."""


def refine_batch_sharded(cdts, thetas=20.0, group=None, engine=None, gather=True, **kw):
    """Batched refinement of independent domains over the ranks of a process
    group, one GPU per rank.

    Every rank receives the same list of domains.  partition_domains assigns
    them to ranks by estimated cost (domain_cost: points and theta); each rank
    refines its share with one call of `engine` (default: the persistent batch
    engine, refine.refine_batch_persistent, on the GPU given by kw["device"],
    else this rank's LOCAL_RANK) and no data moves between GPUs.  With
    gather=True the results are collected on rank 0 and returned there in
    input order, as (list of CDT, list of stats dicts, report); the other ranks
    return (None, None, report).  With gather=False every rank returns only its
    own share: (its domain ids, its results, its stats, report).

    The gather copies raw arrays through host memory: when all ranks run on
    one node, each rank writes its meshes into one file in /dev/shm and rank 0
    reads them back (no pickling of the meshes); across nodes the shares go
    through gather_object.

    If the engine raises on any rank, every rank still takes part in the same
    collectives and then raises ShardError (naming the failed ranks), so no
    rank is left waiting in a collective.

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
    device = _reduce_device(group, kw.get("device"))
    t0 = time.perf_counter()
    res, stats, failure = [], [], ""
    try:
        if mine:
            res, stats = engine([cdts[i] for i in mine], [th[i] for i in mine], **kw)
    except Exception as e:  # reported to every rank through the reduction below
        failure = f"{type(e).__name__}: {e}"
    rank_ms = (time.perf_counter() - t0) * 1e3
    # one reduction carries the job time and whether any rank failed
    max_ms, failed = _reduce_time_and_failure(rank_ms, bool(failure), group, device)
    report = {"rank_ms": rank_ms, "max_ms": max_ms, "domains": [len(p) for p in parts], "loads": loads}
    if failed:
        raise ShardError(f"the batch engine failed on {failed} rank(s)" + (f"; here: {failure}" if failure else ""))
    if not gather:
        return mine, res, stats, report
    got = _gather_shares(mine, list(res), list(stats), rank, world, group, on)
    if rank != 0:
        return None, None, report
    out, out_stats = [None] * n, [None] * n
    for ids, r, s in got:
        for i, a, b in zip(ids, r, s):
            out[i], out_stats[i] = a, b
    return out, out_stats, report


def _reduce_time_and_failure(local_ms, failed, group, device):
    """(max of local_ms over ranks, number of ranks that failed)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(local_ms), 1.0 if failed else 0.0], dtype=torch.float64, device=device)
    f = t[1:].clone()
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(f, op=dist.ReduceOp.SUM, group=group)
    return float(t[0].item()), int(round(float(f[0].item())))


FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _pack(res):
    """Meshes -> one byte buffer: per mesh its three sizes, then its arrays."""
    import numpy as np

    parts = [np.asarray([len(res)], np.int64).view(np.uint8)]
    for c in res:
        parts.append(np.asarray([c.numberofpoints, c.numberoftriangles, c.numberofsegments], np.int64).view(np.uint8))
        for f in FIELDS:
            parts.append(np.ascontiguousarray(getattr(c, f)).view(np.uint8).reshape(-1))
    return np.concatenate(parts) if parts else np.zeros(0, np.uint8)


def _unpack(buf):
    import numpy as np

    from .cdtio import CDT
    off = 0

    def take(dtype, count):
        nonlocal off
        nb = np.dtype(dtype).itemsize * count
        a = buf[off:off + nb].view(dtype).copy()
        off += nb
        return a

    out = []
    for _ in range(int(take(np.int64, 1)[0])):
        npt, ntr, nsg = (int(x) for x in take(np.int64, 3))
        out.append(CDT(take(np.float64, 2 * npt), take(np.int32, 3 * ntr), take(np.int32, 3 * ntr),
                       take(np.int32, 2 * nsg)))
    return out


def _gather_shares(ids, res, stats, rank, world, group, on):
    """[(ids, meshes, stats) of every rank] on rank 0 (None elsewhere)."""
    import os
    import socket
    import tempfile

    import numpy as np
    import torch.distributed as dist

    if not on or world == 1:
        return [(ids, res, stats)]
    dst = dist.get_global_rank(group, 0) if group is not None else 0
    hosts = [None] * world
    dist.all_gather_object(hosts, socket.gethostname(), group=group)
    if len(set(hosts)) > 1:  # ranks on several nodes: the shares travel through the process group
        got = [None] * world if rank == 0 else None
        dist.gather_object((ids, res, stats), got, dst=dst, group=group)
        return got
    shm = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    token = [os.urandom(8).hex() if rank == 0 else None]
    dist.broadcast_object_list(token, src=dst, group=group)
    path = os.path.join(shm, f"gqm_shard_{token[0]}_{rank}")
    buf = _pack(res)
    with open(path, "wb") as f:
        f.write(buf.tobytes())
    # ids and stats are small: they go through the process group
    meta = [None] * world if rank == 0 else None
    dist.gather_object((ids, stats), meta, dst=dst, group=group)  # also orders the writes before the reads
    got = None
    try:
        if rank == 0:
            got = []
            for r in range(world):
                data = np.fromfile(os.path.join(shm, f"gqm_shard_{token[0]}_{r}"), dtype=np.uint8)
                got.append((meta[r][0], _unpack(data), meta[r][1]))
    finally:
        dist.barrier(group=group)  # rank 0 has read every file
        os.remove(path)
    return got


def _reduce_device(group, device=None):
    """Device of the reduction tensors: under NCCL the GPU this rank's engine
    runs on (`device`, else the current CUDA device), the host otherwise."""
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_backend(group) == "nccl":
        return torch.device("cuda", int(device) if device is not None else torch.cuda.current_device())
    return None
