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
    domain (the CUDA engine is held to the same outputs by the GPU tests).  The
    emulated-engine tests below run the engine's own code instead."""
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


# --- the engine's own code on CPU ranks --------------------------------------

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU_LIB = os.path.join(ROOT, "tests", "emu", "_build", "libgqm_emu.so")


def _emu_worker(rank, world, port, out, fail_rank):
    """A gloo rank whose engine is the persistent batch engine of this
    repository (batch.cu and refine.cu compiled as host C++ against the
    test-only runtime stand-in, tests/emu); with fail_rank set, that rank's
    engine raises instead."""
    import pickle

    import torch.distributed as dist
    from gpu_cdt_refine_b200 import refine
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    refine.use_library(EMU_LIB)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        doms, thetas = _shard_domains()
        engine = None
        if fail_rank == rank:
            def engine(d, t, **kw):
                raise RuntimeError("injected engine failure")
        try:
            res, stats, rep = replicas.refine_batch_sharded(doms, thetas, engine=engine, device=0)
            out[rank] = pickle.dumps(("ok", res, rep))
        except replicas.ShardError as e:
            out[rank] = pickle.dumps(("failed", str(e), None))
        # the process group still works after a failed call on every rank
        ms, _ = replicas.reduce_step(1.0 + rank, 0.0)
        out[f"after{rank}"] = ms
    finally:
        dist.destroy_process_group()


def _build_emu():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "tests", "emu"), EMU_LIB])


def test_batch_sharded_emulated_engine_matches_oracle():
    """Two gloo ranks run the persistent batch engine's own code (emulated on
    the host) on their shares; rank 0 gathers the raw arrays through /dev/shm,
    in input order, equal to the oracle byte for byte."""
    import pickle

    import numpy as np
    _build_emu()
    mgr = mp.Manager()
    out = mgr.dict()
    port = 30100 + (os.getpid() % 1000)
    mp.spawn(_emu_worker, args=(2, port, out, -1), nprocs=2, join=True)
    doms, thetas = _shard_domains()
    want, _ = _oracle_engine(doms, thetas)
    kind0, res0, rep0 = pickle.loads(out[0])
    kind1, res1, _ = pickle.loads(out[1])
    assert kind0 == kind1 == "ok" and res1 is None
    assert sorted(rep0["domains"]) == [3, 3] or sum(rep0["domains"]) == len(doms)
    for g, w in zip(res0, want):
        for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
            assert np.array_equal(getattr(g, f).view(np.uint8), getattr(w, f).view(np.uint8)), f
    assert out["after0"] == out["after1"] == 2.0


@pytest.mark.parametrize("fail_rank", [0, 1])
def test_batch_sharded_engine_failure_reaches_every_rank(fail_rank):
    """One rank's engine raises: both ranks raise ShardError after the same
    collectives (none waits for the process-group timeout), and the group is
    still usable."""
    import pickle
    _build_emu()
    mgr = mp.Manager()
    out = mgr.dict()
    port = 30300 + 10 * fail_rank + (os.getpid() % 1000)
    mp.spawn(_emu_worker, args=(2, port, out, fail_rank), nprocs=2, join=True)
    for r in range(2):
        kind, msg, _ = pickle.loads(out[r])
        assert kind == "failed" and "1 rank(s)" in msg
        assert ("injected engine failure" in msg) == (r == fail_rank)
    assert out["after0"] == out["after1"] == 2.0


def test_pack_unpack_roundtrip():
    import numpy as np
    doms, _ = _shard_domains()
    back = replicas._unpack(replicas._pack(doms[:3]))
    for a, b in zip(back, doms[:3]):
        for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
            assert np.array_equal(getattr(a, f), getattr(b, f))
    assert replicas._unpack(replicas._pack([])) == []
