"""Parity of the sm_100a refiner with the oracle, bit for bit, through the C ABI.

Every output array (points, triangles, neighbours, segments, status bytes) is
compared byte for byte: the slot assignment, compaction order and FP64
arithmetic of the reference are reproduced, not only the mesh."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from gpu_cdt_refine_b200.certify import certify
from oracle import oracle_py

pytestmark = pytest.mark.gpu

CFGS = [(20.0, 1, 1), (20.0, 1, 0), (20.0, 0, 1), (20.0, 0, 0)]
FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def assert_same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape, (f, x.shape, y.shape)
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f


@pytest.fixture(scope="module")
def small_inputs():
    return {
        "u2k": inputs.plain_small(seed=201, n=2000, nseg=100),
        "u5k_dense_segs": inputs.plain_small(seed=202, n=5000, nseg=600),
        "cl8k": inputs.clustered(seed=203, n=8000, nseg=400),
    }


@pytest.mark.parametrize("theta,policy,mode", CFGS)
@pytest.mark.parametrize("case", ["u2k", "u5k_dense_segs", "cl8k"])
def test_matches_oracle(gpu, small_inputs, case, theta, policy, mode):
    cdt = small_inputs[case]
    got, ps, ts, st = refine.refine(cdt, theta, policy, mode, with_status=True)
    want, info = oracle_py.refine(cdt, theta, policy, mode)
    assert st["rounds"] == info["rounds"]
    assert_same(got, want)
    assert np.array_equal(ps, info["pstatus"])
    assert np.array_equal(ts, info["tstatus"])


def test_c1_workload_matches_oracle(gpu):
    """10,000 uniform points, 500 segments, theta 20, Ruppert, Offcenter."""
    cdt = inputs.plain_small()
    got, st = refine.refine(cdt, 20.0, refine.Offcenter, 1)
    want, info = oracle_py.refine(cdt, 20.0, 1, 1)
    assert_same(got, want)
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert


@pytest.mark.parametrize("theta", [15.0, 18.0, 25.0])
def test_other_angles(gpu, small_inputs, theta):
    cdt = small_inputs["u2k"]
    got, st = refine.refine(cdt, theta, refine.Offcenter, 1)
    want, _ = oracle_py.refine(cdt, theta, 1, 1)
    assert_same(got, want)


def test_device_cos_reported(gpu, small_inputs):
    _, st = refine.refine(small_inputs["u2k"], 20.0)
    c = np.cos(20.0 * np.pi / 180.0)
    assert st["goodcos2"] == c * c


def test_exact_predicates_certify(gpu, small_inputs):
    cdt = small_inputs["cl8k"]
    got, st = refine.refine(cdt, 20.0, refine.Offcenter, 1, predicates=refine.PRED_EXACT)
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert


def test_context_reuse_is_deterministic(gpu, small_inputs):
    ctx = refine.Context(0)
    opt = refine.make_options(20.0, refine.Offcenter, 1)
    ctx.run_host(small_inputs["cl8k"], opt)
    a = ctx.result()
    ctx.run_host(small_inputs["u2k"], opt)
    ctx.run_host(small_inputs["cl8k"], opt)
    b = ctx.result()
    ctx.close()
    assert_same(a, b)


def test_round_limit_returns_status(gpu, small_inputs):
    with pytest.raises(refine.RefineError) as e:
        refine.refine(small_inputs["u2k"], 20.0, max_rounds=1)
    assert e.value.status == -2


@pytest.mark.parametrize("area", [50.0, 400.0])
def test_area_bound_matches_oracle(gpu, area):
    """Area bound (Triangle's `a` switch; no counterpart in the reference):
    CUDA path == oracle byte for byte, every triangle within the bound."""
    cdt = inputs.plain_small(seed=361, n=5000, nseg=200)
    got, _ = refine.refine(cdt, 20.0, max_area=area)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1, max_area=area)
    assert_same(got, want)
    t = got.pointlist[got.trianglelist]
    a = 0.5 * np.abs((t[:, 1, 0] - t[:, 0, 0]) * (t[:, 2, 1] - t[:, 0, 1]) -
                     (t[:, 1, 1] - t[:, 0, 1]) * (t[:, 2, 0] - t[:, 0, 0]))
    assert a.max() <= area
    gb, _ = refine.refine_batch_persistent([cdt], 20.0, max_area=area)
    assert_same(gb[0], got)


def test_domain_with_hole_matches_oracle(gpu):
    cdt = inputs.square_with_hole(n=8000)
    got, _ = refine.refine(cdt, 20.0)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    assert_same(got, want)
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert
