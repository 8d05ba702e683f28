"""Constrained Delaunay triangulation on the GPU (csrc/cdt_gpu.cu).

``build_cdt_gpu(points, segments)`` returns the same :class:`CDT` as
``inputs.build_cdt`` (the exact CPU builder): the input of the refiner in
Triangle's "pzQnc" layout (GPU_Refine/mesh.cpp:397), with the convex hull
enclosed by segments.  For points with no four cocircular the triangulation is
unique and both builders agree up to numbering (``cdtio.same_mesh``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native, refine
from .cdtio import CDT


class CdtGpuStats(ctypes.Structure):
    _fields_ = [("hull_vertices", ctypes.c_int), ("hull_candidates", ctypes.c_int),
                ("insert_rounds", ctypes.c_int), ("flip_rounds", ctypes.c_int),
                ("recover_rounds", ctypes.c_int), ("segments_missing", ctypes.c_int),
                ("flips", ctypes.c_longlong), ("recover_flips", ctypes.c_longlong),
                ("kernel_launches", ctypes.c_longlong),
                ("ms_h2d", ctypes.c_double), ("ms_hull", ctypes.c_double), ("ms_insert", ctypes.c_double),
                ("ms_segments", ctypes.c_double), ("ms_output", ctypes.c_double), ("ms_d2h", ctypes.c_double),
                ("ms_total", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


STATUS = {-1: "fewer than 3 points", -2: "all points collinear", -4: "bad segment index",
          -6: "segments cross", -7: "a point lies on a segment", -8: "duplicate points",
          -9: "internal invariant failed", -10: "CUDA error", -11: "out of device memory",
          -12: "no such device"}


class CdtBuildError(RuntimeError):
    def __init__(self, status: int):
        super().__init__(f"GPU CDT construction failed: {STATUS.get(status, status)} ({status})")
        self.status = status


def _bind():
    L = refine.lib()
    if not getattr(L, "_cdt_bound", False):
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.gqm_cdt_build_gpu.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ctypes.c_int,
                                        ctypes.POINTER(_native.CdtResult), ctypes.POINTER(CdtGpuStats)]
        L.gqm_cdt_build_gpu.restype = ctypes.c_int
        L.gqm_cdt_gpu_free.argtypes = [ctypes.POINTER(_native.CdtResult)]
        L.gqm_cdt_gpu_release.argtypes = []
        L._cdt_bound = True
    return L


def build_cdt_gpu(points: np.ndarray, segments: np.ndarray, device: int = 0, with_stats: bool = False):
    """CDT of the points and segments, convex hull enclosed by segments."""
    L = _bind()
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    seg = np.ascontiguousarray(segments, dtype=np.int32).reshape(-1, 2)
    res = _native.CdtResult()
    st = CdtGpuStats()
    rc = L.gqm_cdt_build_gpu(pts.shape[0], _native.dptr(pts), seg.shape[0], _native.iptr(seg), device, res, st)
    if rc != 0:
        raise CdtBuildError(rc)
    try:
        t, s = res.numberoftriangles, res.numberofsegments
        tri = np.ctypeslib.as_array(res.trianglelist, shape=(t * 3,)).copy()
        nbr = np.ctypeslib.as_array(res.neighborlist, shape=(t * 3,)).copy()
        sg = np.ctypeslib.as_array(res.segmentlist, shape=(s * 2,)).copy() if s else np.zeros(0, np.int32)
    finally:
        L.gqm_cdt_gpu_free(res)
    cdt = CDT(pts.copy(), tri, nbr, sg)
    return (cdt, st.as_dict()) if with_stats else cdt


def release() -> None:
    """Frees the device buffers the builder keeps between calls."""
    _bind().gqm_cdt_gpu_release()
