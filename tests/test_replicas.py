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
