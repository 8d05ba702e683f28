"""The refiner's own kernels and driver (csrc/refine.cu), compiled as host
C++ against a test-only runtime stand-in (tests/emu), agree with the oracle
byte for byte.  This checks the kernels' index arithmetic and bookkeeping on a
machine without a GPU; the GPU parity tests repeat the comparison on a B200."""
import os
import subprocess

import numpy as np
import pytest

from gpu_cdt_refine_b200 import _native, inputs, refine
from oracle import oracle_py

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "emu")
FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _emu_lib(name):
    path = os.path.join(EMU, "_build", name)
    subprocess.check_call(["make", "-s", "-C", EMU, path])
    return path


@pytest.fixture()
def emulated(request):
    saved_path, saved_lib = _native.CUDA_LIB, refine._lib
    _native.CUDA_LIB = _emu_lib(getattr(request, "param", "libgqm_emu.so"))
    refine._lib = None
    yield
    _native.CUDA_LIB, refine._lib = saved_path, saved_lib


def _same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f


@pytest.mark.parametrize("theta,policy,mode", [(20.0, 1, 1), (20.0, 1, 0), (20.0, 0, 1), (20.0, 0, 0), (15.0, 1, 1)])
def test_emulated_matches_oracle(emulated, theta, policy, mode):
    cdt = inputs.plain_small(seed=301, n=3000, nseg=200)
    got, ps, ts, st = refine.refine(cdt, theta, policy, mode, with_status=True)
    want, info = oracle_py.refine(cdt, theta, policy, mode)
    _same(got, want)
    assert np.array_equal(ps, info["pstatus"]) and np.array_equal(ts, info["tstatus"])
    assert st["rounds"] == info["rounds"]


@pytest.mark.parametrize("emulated", ["libgqm_emu_tight.so"], indirect=True)
def test_emulated_buffer_regrowth(emulated):
    """Physical buffers sized exactly to the logical capacity: every growth
    step reallocates and copies, and the result is unchanged."""
    cdt = inputs.clustered(seed=302, n=20000, nseg=1000)
    got, _ = refine.refine(cdt, 20.0, 1, 1)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    _same(got, want)


def test_emulated_round_limit(emulated):
    cdt = inputs.plain_small(seed=303, n=1000, nseg=50)
    with pytest.raises(refine.RefineError) as e:
        refine.refine(cdt, 20.0, max_rounds=1)
    assert e.value.status == -2


@pytest.mark.parametrize("field,row,col,value", [
    ("segmentlist", 0, 0, 10**6),   # segment endpoint out of range
    ("segmentlist", 1, 1, -4),      # negative endpoint
    ("trianglelist", 5, 2, 10**6),  # triangle vertex out of range
    ("neighborlist", 7, 0, 10**7),  # neighbour index out of range
])
def test_emulated_rejects_bad_indices(emulated, field, row, col, value):
    """Out-of-range indices are caught on the device before any kernel reads
    through them (GQM_ERR_ARGUMENT)."""
    cdt = inputs.plain_small(seed=304, n=500, nseg=20)
    arr = getattr(cdt, field).copy()
    arr.reshape(-1, arr.shape[-1])[row, col] = value
    setattr(cdt, field, arr)
    with pytest.raises(refine.RefineError) as e:
        refine.refine(cdt, 20.0)
    assert e.value.status == -1


def test_emulated_batch(emulated):
    doms = [inputs.plain_small(seed=310 + i, n=n, nseg=n // 20) for i, n in enumerate([300, 1500, 700])]
    got, stats = refine.refine_batch(doms, [15.0, 20.0, 18.0], workers=2)
    for d, th, g, st in zip(doms, [15.0, 20.0, 18.0], got, stats):
        want, info = oracle_py.refine(d, th, 1, 1)
        _same(g, want)
        assert st["rounds"] == info["rounds"]


def _persistent_domains():
    doms = [inputs.plain_small(seed=320 + i, n=n, nseg=max(4, n // 20)) for i, n in enumerate([300, 1500, 700, 2500])]
    doms.append(inputs.clustered(seed=329, n=2000, nseg=100))
    return doms


def test_emulated_persistent_batch_matches_oracle(emulated):
    """The persistent batch engine (csrc/batch.cu: one block refines a whole
    domain, the driver running on the device) gives each domain the oracle's
    result byte for byte, for mixed angles, modes and insertion policies."""
    doms = _persistent_domains()
    cfg = [(15.0, 1, 1), (20.0, 1, 0), (18.0, 0, 1), (20.0, 0, 0), (20.0, 1, 1)]
    for (theta, policy, mode), d in zip(cfg, doms):
        got, st = refine.refine_batch_persistent([d], theta, policy, mode)
        want, info = oracle_py.refine(d, theta, policy, mode)
        _same(got[0], want)
        assert st[0]["rounds"] == info["rounds"]
    got, st, rep = refine.refine_batch_persistent(doms, [c[0] for c in cfg], with_report=True)
    assert rep["fallbacks"] == 0
    for (theta, _, _), d, g in zip(cfg, doms, got):
        want, _ = oracle_py.refine(d, theta, 1, 1)
        _same(g, want)


def test_emulated_persistent_batch_exact_predicates(emulated):
    """Domains with exact predicates run in their own persistent launch and
    match the single-domain path with exact predicates."""
    doms = _persistent_domains()[:3]
    preds = [refine.PRED_EXACT, refine.PRED_REFERENCE, refine.PRED_EXACT]
    got, _ = refine.refine_batch_persistent(doms, 20.0, predicates=preds)
    for d, p, g in zip(doms, preds, got):
        one, _ = refine.refine(d, 20.0, predicates=p)
        _same(g, one)


@pytest.mark.parametrize("emulated", ["libgqm_emu_tight.so"], indirect=True)
def test_emulated_persistent_batch_arena_fallback(emulated):
    """Arenas with no room to grow: domains that outgrow them are refined again
    by the single-domain path, and every result is still the oracle's."""
    doms = _persistent_domains()
    got, _, rep = refine.refine_batch_persistent(doms, 20.0, with_report=True)
    assert rep["fallbacks"] > 0
    for d, g in zip(doms, got):
        want, _ = oracle_py.refine(d, 20.0, 1, 1)
        _same(g, want)
