"""The C-ABI libraries load and export every function the headers declare."""
import ctypes
import os
import re

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
