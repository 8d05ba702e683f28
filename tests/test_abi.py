"""The C-ABI libraries load and export every function the headers declare."""
import ctypes
import os
import re

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
