"""The oracle (CPU restatement of refine.cu) on small inputs: every output is
a certified constrained Delaunay triangulation with minimum angle >= theta,
and the run is deterministic."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import cdtio, inputs
from gpu_cdt_refine_b200.certify import certify
from oracle import oracle_py

CFGS = [(20.0, 1, 1), (20.0, 1, 0), (20.0, 0, 1), (20.0, 0, 0), (15.0, 1, 1), (18.0, 1, 1)]


@pytest.fixture(scope="module")
def small():
    return inputs.plain_small(seed=101, n=2000, nseg=100)


@pytest.mark.parametrize("theta,policy,mode", CFGS)
def test_oracle_output_certifies(small, theta, policy, mode):
    out, info = oracle_py.refine(small, theta, policy, mode)
    cert = certify(out, small, theta)
    assert cert["ok"], cert
    assert cert["triangles_below_theta"] == 0, cert
    assert cert["min_angle_deg"] >= theta
    assert info["rounds"] > 0


def test_oracle_deterministic(small):
    a, _ = oracle_py.refine(small, 20.0, 1, 1)
    b, _ = oracle_py.refine(small, 20.0, 1, 1)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(a, f), getattr(b, f))


def test_oracle_offconstant_is_truncated():
    """offconstant is passed to splitTriangles as an int (refine.cu:5132):
    at theta=20 it is 2, so circumcentres farther than the off-centre at
    2 x shortest edge are replaced."""
    L = oracle_py.lib()
    import ctypes
    DP = ctypes.POINTER(ctypes.c_double)
    apex = np.array([0.0, 10.0]); org = np.array([0.0, 0.0]); dest = np.array([1.0, 0.0])
    out = np.zeros(2)
    L.gqm_oracle_circumcenter(apex.ctypes.data_as(DP), org.ctypes.data_as(DP), dest.ctypes.data_as(DP), 2.0, 1,
                              out.ctypes.data_as(DP))
    # shortest edge org-dest: off-centre at midpoint + 2 * |od| along the bisector
    assert out[0] == 0.5 and out[1] == 2.0


def test_oracle_input_points_preserved(small):
    out, _ = oracle_py.refine(small, 20.0, 1, 1)
    n = small.numberofpoints
    assert np.array_equal(out.pointlist[:n], small.pointlist)
