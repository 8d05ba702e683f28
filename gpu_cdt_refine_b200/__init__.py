"""B200-native constrained Delaunay quality refinement.

The drop-in entry point mirrors the reference's
``GPU_Refine_Quality(triangulateio*, triangulateio*, theta, InsertPolicy,
DeletePolicy, mode, debug_iter, ps_debug, ts_debug)`` (GPU_Refine/refine.h:385-386)
and runs hand-written sm_100a CUDA through the C ABI in include/gqm_refine.h.
"""
from .cdtio import CDT, read_cdt, write_cdt, canonical, same_mesh  # noqa: F401

Circumcenter = 0
Offcenter = 1
