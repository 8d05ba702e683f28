"""Multi-rank host logic on CPU with gloo (world size 2)."""
import os

import pytest
import torch.multiprocessing as mp

from gpu_cdt_refine_b200 import replicas


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, tris = replicas.reduce_step(10.0 + 5.0 * rank, 1000.0 * (rank + 1))
        out[rank] = (ms, tris)
    finally:
        dist.destroy_process_group()


def test_reduce_step_two_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() % 1000)
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (15.0, 3000.0)


def test_reduce_step_single_process():
    assert replicas.reduce_step(3.0, 7.0) == (3.0, 7.0)


def test_partition_domains_balanced_and_complete():
    costs = [replicas.domain_cost(n, th) for n, th in
             zip([200, 50000, 3000, 12000, 800, 45000, 7000, 20000], [15, 20, 18, 20, 15, 18, 20, 15])]
    parts, loads = replicas.partition_domains(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    assert max(loads) <= sum(costs) / 3 + max(costs)


def test_partition_domains_deterministic():
    costs = [float(c) for c in (5, 5, 5, 5, 1)]
    assert replicas.partition_domains(costs, 2) == replicas.partition_domains(costs, 2)


# --- batched domains sharded over ranks (replicas.refine_batch_sharded) -------

def _oracle_engine(doms, thetas, **kw):
    """Stand-in for the persistent batch engine on CPU ranks: the oracle on each
    domain (the CUDA engine is held to the same outputs by the GPU tests)."""
    from oracle import oracle_py
    outs = [oracle_py.refine(d, t, 1, 1) for d, t in zip(doms, thetas)]
    return [o[0] for o in outs], [o[1] for o in outs]


def _shard_domains():
    from gpu_cdt_refine_b200 import inputs
    sizes = [300, 1200, 500, 900, 250, 700]
    doms = [inputs.plain_small(seed=960 + i, n=n, nseg=max(4, n // 25)) for i, n in enumerate(sizes)]
    return doms, [15.0, 20.0, 18.0, 20.0, 15.0, 18.0]


def _shard_worker(rank, world, port, out, count=None):
    import pickle

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        doms, thetas = _shard_domains()
        doms, thetas = doms[:count], thetas[:count]
        res, stats, rep = replicas.refine_batch_sharded(doms, thetas, engine=_oracle_engine)
        ids, own, _, rep2 = replicas.refine_batch_sharded(doms, thetas, engine=_oracle_engine, gather=False)
        out[rank] = pickle.dumps((res, stats, rep, ids, own, rep2))
    finally:
        dist.destroy_process_group()


def test_batch_sharded_two_ranks_matches_unsharded():
    import pickle

    import numpy as np
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = 29700 + (os.getpid() % 1000)
    mp.spawn(_shard_worker, args=(world, port, out), nprocs=world, join=True)
    doms, thetas = _shard_domains()
    want, _ = _oracle_engine(doms, thetas)
    res0, st0, rep0, ids0, own0, _ = pickle.loads(out[0])
    res1, st1, rep1, ids1, own1, _ = pickle.loads(out[1])
    assert res1 is None and st1 is None
    assert rep0["max_ms"] == rep1["max_ms"] >= max(rep0["rank_ms"], rep1["rank_ms"]) - 1e-9
    assert rep0["domains"] == [len(ids0), len(ids1)] and sorted(ids0 + ids1) == list(range(len(doms)))
    assert len(res0) == len(doms)
    for g, w in zip(res0, want):  # gathered in input order, byte for byte
        for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
            assert np.array_equal(getattr(g, f).view(np.uint8), getattr(w, f).view(np.uint8))
    for ids, own in ((ids0, own0), (ids1, own1)):  # gather=False: each rank keeps its own share
        for i, g in zip(ids, own):
            assert np.array_equal(g.trianglelist, want[i].trianglelist)


def test_batch_sharded_single_process():
    doms, thetas = _shard_domains()
    res, stats, rep = replicas.refine_batch_sharded(doms[:3], thetas[:3], engine=_oracle_engine)
    want, _ = _oracle_engine(doms[:3], thetas[:3])
    assert rep["domains"] == [3]
    assert all(a.numberoftriangles == b.numberoftriangles for a, b in zip(res, want))


def test_batch_sharded_rank_without_domains():
    """One domain over two ranks: the rank that receives none takes part in
    the timing reduction and the gather, and rank 0 returns the one result."""
    import pickle
    mgr = mp.Manager()
    out = mgr.dict()
    port = 29900 + (os.getpid() % 1000)
    mp.spawn(_shard_worker, args=(2, port, out, 1), nprocs=2, join=True)
    doms, thetas = _shard_domains()
    want, _ = _oracle_engine(doms[:1], thetas[:1])
    res0, _, rep0, ids0, _, _ = pickle.loads(out[0])
    res1, _, rep1, ids1, _, _ = pickle.loads(out[1])
    assert sorted(rep0["domains"]) == [0, 1] and res1 is None
    assert sorted(ids0 + ids1) == [0]
    assert len(res0) == 1 and res0[0].numberoftriangles == want[0].numberoftriangles
