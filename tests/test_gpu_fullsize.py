"""The benchmark workload at full size (2,000,000 clustered points, 100,000
segments, theta 20, Ruppert, Offcenter) through the C ABI: size-independent
properties (exact certificate, minimum angle, determinism, input points
preserved), plus a bit-for-bit oracle comparison at 500,000 points."""
import hashlib

import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from gpu_cdt_refine_b200.certify import certify
from oracle import oracle_py

pytestmark = pytest.mark.gpu


def _digest(c):
    h = hashlib.sha256()
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        h.update(np.ascontiguousarray(getattr(c, f)).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def workload():
    return inputs.clustered()


def test_fullsize_certified_and_deterministic(gpu, workload):
    a, st = refine.refine(workload, 20.0, refine.Offcenter, 1)
    b, _ = refine.refine(workload, 20.0, refine.Offcenter, 1)
    assert _digest(a) == _digest(b)
    cert = certify(a, workload, 20.0)
    assert cert["ok"], cert
    assert cert["triangles_below_theta"] == 0 and cert["min_angle_deg"] >= 20.0
    assert cert["max_segment_deviation"] < 1e-9
    assert a.numberoftriangles > 2 * workload.numberoftriangles


def test_500k_matches_oracle(gpu):
    cdt = inputs.clustered(seed=31, n=500_000, nseg=25_000)
    got, st = refine.refine(cdt, 20.0, refine.Offcenter, 1)
    want, info = oracle_py.refine(cdt, 20.0, 1, 1)
    assert st["rounds"] == info["rounds"]
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        x, y = getattr(got, f), getattr(want, f)
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), f
