"""Loading of the in-tree native libraries.

``libgqm_host.so``  : CPU side (CDT construction, synthetic inputs, certificate)
``libgqm_b200.so``  : the sm_100a refiner behind the C ABI of include/gqm_refine.h

Both are built in-tree by :mod:`gpu_cdt_refine_b200.build`.  Loading fails
loudly when a library is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB = os.path.join(HERE, "libgqm_host.so")
CUDA_LIB = os.path.join(HERE, "libgqm_b200.so")

_host = None
_cuda = None


class CdtResult(ctypes.Structure):
    _fields_ = [("numberofpoints", ctypes.c_int), ("numberoftriangles", ctypes.c_int),
                ("numberofsegments", ctypes.c_int), ("status", ctypes.c_int),
                ("trianglelist", ctypes.POINTER(ctypes.c_int)),
                ("neighborlist", ctypes.POINTER(ctypes.c_int)),
                ("segmentlist", ctypes.POINTER(ctypes.c_int))]


def host() -> ctypes.CDLL:
    global _host
    if _host is None:
        if not os.path.exists(HOST_LIB):
            raise RuntimeError(f"{HOST_LIB} is missing: run gpu_cdt_refine_b200.build first")
        lib = ctypes.CDLL(HOST_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.gqm_cdt_build.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ctypes.POINTER(CdtResult)]
        lib.gqm_cdt_build.restype = ctypes.c_int
        lib.gqm_cdt_free.argtypes = [ctypes.POINTER(CdtResult)]
        lib.gqm_synth_uniform.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, dp]
        lib.gqm_synth_uniform.restype = ctypes.c_int
        lib.gqm_synth_clusters.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_uint64, dp]
        lib.gqm_synth_clusters.restype = ctypes.c_int
        lib.gqm_synth_grid_circles.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_uint64, dp, ip]
        lib.gqm_synth_grid_circles.restype = ctypes.c_int
        lib.gqm_pick_segments.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                          ctypes.c_longlong, ip]
        lib.gqm_pick_segments.restype = ctypes.c_int
        lib.gqm_filter_segments.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ctypes.c_int, ip]
        lib.gqm_filter_segments.restype = ctypes.c_int
        lib.gqm_remove_holes.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ctypes.c_int, dp,
                                         ctypes.c_void_p]
        lib.gqm_remove_holes.restype = ctypes.c_int
        lib.gqm_region_attributes.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ctypes.c_int,
                                              dp, dp, dp]
        lib.gqm_region_attributes.restype = ctypes.c_int
        lib.gqm_mesh_free.argtypes = [ctypes.c_void_p]
        if hasattr(lib, "gqm_certify"):
            lib.gqm_certify.restype = ctypes.c_int
        _host = lib
    return _host


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
