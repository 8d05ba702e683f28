"""The C-ABI libraries load and export every function the headers declare."""
import ctypes
import os
import re

import numpy as np
import pytest

from gpu_cdt_refine_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gqm_[a-z_0-9]+)\s*\(", text)))


def test_cuda_library_exports_header_functions():
    lib = ctypes.CDLL(_native.CUDA_LIB)
    names = _declared("gqm_refine.h")
    assert "gqm_refine" in names and "gqm_context_run" in names
    for n in names:
        assert hasattr(lib, n), n


def test_cpp_drop_in_symbol_matches_reference_mangling():
    # GPU_Refine_Quality(triangulateio*, triangulateio*, double, InsertPolicy,
    # DeletePolicy, int, int, PStatus**, TStatus**) -- refine.h:385-386
    lib = ctypes.CDLL(_native.CUDA_LIB)
    assert hasattr(lib, "_Z18GPU_Refine_QualityP13triangulateioS0_d12InsertPolicy12DeletePolicyiiPP7PStatusPP7TStatus")


def test_status_strings_and_no_device_error():
    from gpu_cdt_refine_b200 import refine
    L = refine.lib()
    assert L.gqm_status_string(0) == b"ok"
    assert L.gqm_version() >= 100


def _bad_call(case):
    """gqm_refine on a small valid CDT with one argument made invalid."""
    from gpu_cdt_refine_b200 import inputs, refine
    L = refine.lib()
    cdt = inputs.plain_small(seed=11, n=200, nseg=10)
    keep = []
    cin = refine._cdt_in(cdt, keep)
    opt = refine.make_options(20.0, refine.Offcenter, 1)
    if case == "few_points":
        cin.numberofpoints = 2
    elif case == "no_triangles":
        cin.numberoftriangles = 0
    elif case == "negative_segments":
        cin.numberofsegments = -1
    elif case == "null_points":
        cin.pointlist = None
    elif case == "null_neighbours":
        cin.neighborlist = None
    elif case == "null_segments":
        cin.segmentlist = None
    elif case in ("theta_zero", "theta_60", "theta_nan"):
        opt.theta = {"theta_zero": 0.0, "theta_60": 60.0, "theta_nan": float("nan")}[case]
    elif case == "negative_area":
        opt.max_area = -1.0
    elif case == "learned_without_network":
        opt.placement = refine.PLACE_LEARNED
        opt.mlp = None
    out = refine.CdtOut()
    if case == "null_input":
        return L.gqm_refine(None, ctypes.byref(out), ctypes.byref(opt), None)
    if case == "null_output":
        return L.gqm_refine(ctypes.byref(cin), None, ctypes.byref(opt), None)
    rc = L.gqm_refine(ctypes.byref(cin), ctypes.byref(out), ctypes.byref(opt), None)
    assert not out.pointlist and not out.trianglelist  # nothing handed out on an error
    return rc


@pytest.mark.parametrize("case", ["null_input", "null_output", "few_points", "no_triangles", "negative_segments",
                                  "null_points", "null_neighbours", "null_segments", "theta_zero", "theta_60",
                                  "theta_nan", "negative_area", "learned_without_network"])
def test_refine_rejects_invalid_arguments_before_touching_a_device(case):
    """Argument checks run on the host before any CUDA call, so they answer the
    same on a machine without a GPU: GQM_ERR_ARGUMENT, and no output arrays."""
    assert _bad_call(case) == -1


@pytest.mark.parametrize("case", ["null_input", "one_level", "many_levels", "eps_negative", "eps_above_one",
                                  "negative_cap", "null_rows", "theta_zero"])
def test_learn_explore_rejects_invalid_arguments_before_touching_a_device(case):
    """gqm_learn_explore checks its arguments and options on the host first."""
    from gpu_cdt_refine_b200 import inputs, refine
    L = refine.lib()
    cdt = inputs.plain_small(seed=12, n=200, nseg=10)
    keep = []
    cin = refine._cdt_in(cdt, keep)
    opt = refine.make_options(0.0 if case == "theta_zero" else 20.0, refine.Offcenter, 1)
    levels = {"one_level": 1, "many_levels": 65}.get(case, 5)
    eps = {"eps_negative": -0.1, "eps_above_one": 1.5}.get(case, 1.0)
    cap = -1 if case == "negative_cap" else 16
    f = np.zeros((16, refine.MLP_FEATURES), np.float32)
    i = np.zeros(16, np.int32)
    t = np.zeros(16, np.float32)
    u = np.zeros(16, np.uint8)
    ip = ctypes.POINTER(ctypes.c_int)
    cnt = ctypes.c_longlong(0)
    rows = (None,) * 6 if case == "null_rows" else (refine._fp(f), i.ctypes.data_as(ip), refine._fp(t),
                                                    i.ctypes.data_as(ip), u.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                                    i.ctypes.data_as(ip))
    rc = L.gqm_learn_explore(None if case == "null_input" else ctypes.byref(cin), ctypes.byref(opt), levels, 1, None,
                             eps, *rows, cap, ctypes.byref(cnt))
    assert rc == -1


@pytest.mark.parametrize("n,iters,null", [(0, 5, False), (100, 0, False), (100, 5, True)])
def test_mlp_time_rejects_invalid_arguments_before_touching_a_device(n, iters, null):
    from gpu_cdt_refine_b200 import refine
    L = refine.lib()
    p = np.zeros(refine.MLP_PARAMS, np.float32)
    ms = np.zeros(1, np.float32)
    assert L.gqm_mlp_time(0, None if null else refine._fp(p), n, iters, refine._fp(ms)) == -1
