"""Batched refinement of independent domains (gqm_refine_batch): every domain's
result is byte-identical to a single gqm_refine call on it and to the oracle,
whatever the number of host workers sharing the GPU."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from oracle import oracle_py

pytestmark = pytest.mark.gpu

FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _same(a, b):
    return all(
        getattr(a, f).shape == getattr(b, f).shape
        and np.array_equal(getattr(a, f).view(np.uint8), getattr(b, f).view(np.uint8))
        for f in FIELDS
    )


@pytest.fixture(scope="module")
def domains():
    sizes = [400, 3000, 900, 6000, 1500, 250, 4000, 2200]
    doms = [inputs.plain_small(seed=700 + i, n=n, nseg=max(4, n // 25)) for i, n in enumerate(sizes)]
    doms.append(inputs.clustered(seed=799, n=5000, nseg=250))
    return doms


@pytest.mark.parametrize("workers", [1, 4, 16])
def test_batch_matches_single_calls(gpu, domains, workers):
    thetas = [15.0 + (i % 4) * 2.0 for i in range(len(domains))]
    got, stats = refine.refine_batch(domains, thetas, workers=workers)
    assert len(got) == len(domains)
    for d, th, g, st in zip(domains, thetas, got, stats):
        one, st1 = refine.refine(d, th, refine.Offcenter, 1)
        assert _same(g, one)
        assert st["rounds"] == st1["rounds"]


def test_batch_matches_oracle(gpu, domains):
    got, _ = refine.refine_batch(domains, 20.0, workers=8)
    for d, g in zip(domains, got):
        want, _ = oracle_py.refine(d, 20.0, 1, 1)
        assert _same(g, want)


def test_batch_reports_failing_domain(gpu, domains):
    bad = inputs.plain_small(seed=790, n=300, nseg=10)
    bad.segmentlist = bad.segmentlist.copy()
    bad.segmentlist[0, 0] = bad.numberofpoints + 5  # caught by the device-side input check
    with pytest.raises(refine.RefineError) as e:
        refine.refine_batch([domains[0], bad], 20.0, workers=2)
    assert e.value.status == -1 and "domain 1" in str(e.value)


# --- the persistent batch engine (gqm_refine_batch_persistent) ---------------

@pytest.fixture(scope="module")
def mixed_domains():
    doms, thetas = inputs.batch_domains(48, seed=880, nmin=200, nmax=6000)
    return doms, thetas


@pytest.mark.parametrize("variant", [(0, 0), (128, 4), (256, 1), (256, 2), (512, 1)])
def test_persistent_batch_matches_single_calls(gpu, mixed_domains, variant):
    """Every kernel variant gives each domain the single-domain path's result,
    byte for byte."""
    doms, thetas = mixed_domains
    got, stats, rep = refine.refine_batch_persistent(doms, thetas, threads_per_block=variant[0],
                                                     blocks_per_sm=variant[1], with_report=True)
    assert rep["fallbacks"] == 0 and rep["grid"] >= 1
    for d, th, g, st in zip(doms, thetas, got, stats):
        one, st1 = refine.refine(d, th, refine.Offcenter, 1)
        assert _same(g, one)
        assert st["rounds"] == st1["rounds"] and st["flip_steps"] == st1["flip_steps"]


def test_persistent_batch_matches_oracle(gpu, domains):
    got, _ = refine.refine_batch_persistent(domains, 20.0)
    for d, g in zip(domains, got):
        want, _ = oracle_py.refine(d, 20.0, 1, 1)
        assert _same(g, want)


def test_persistent_batch_modes_and_predicates(gpu, domains):
    """Chew mode, the circumcenter policy and exact predicates (run in a
    launch of their own) agree with the single-domain path."""
    preds = [refine.PRED_EXACT if i % 3 == 0 else refine.PRED_REFERENCE for i in range(len(domains))]
    for policy, mode in [(refine.Circumcenter, 0), (refine.Offcenter, 0), (refine.Circumcenter, 1)]:
        got, _ = refine.refine_batch_persistent(domains, 18.0, policy, mode, predicates=preds)
        for d, p, g in zip(domains, preds, got):
            one, _ = refine.refine(d, 18.0, policy, mode, predicates=p)
            assert _same(g, one)


def test_persistent_batch_autotune(gpu, mixed_domains):
    doms, thetas = mixed_domains
    chosen, ms = refine.batch_autotune(doms[:16], thetas[:16])
    assert chosen in refine.batch_variants() and all(v > 0 for v in ms.values())
    got, _, rep = refine.refine_batch_persistent(doms[:16], thetas[:16], with_report=True)
    assert (rep["threads_per_block"], rep["blocks_per_sm"]) == chosen


def test_persistent_batch_reports_failing_domain(gpu, domains):
    bad = inputs.plain_small(seed=791, n=300, nseg=10)
    bad.segmentlist = bad.segmentlist.copy()
    bad.segmentlist[0, 0] = bad.numberofpoints + 5  # caught by the device-side input check
    with pytest.raises(refine.RefineError) as e:
        refine.refine_batch_persistent([domains[0], bad, domains[1]], 20.0)
    assert e.value.status == -1 and "domain 1" in str(e.value)
