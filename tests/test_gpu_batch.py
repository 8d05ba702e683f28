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
