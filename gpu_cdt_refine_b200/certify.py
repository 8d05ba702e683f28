"""Exact certificate of a refined CDT (csrc/certify.cpp)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .cdtio import CDT


class _Cert(ctypes.Structure):
    _fields_ = [("not_ccw", ctypes.c_longlong), ("bad_neighbors", ctypes.c_longlong),
                ("open_boundary", ctypes.c_longlong), ("non_delaunay", ctypes.c_longlong),
                ("segments_missing", ctypes.c_longlong), ("input_points_moved", ctypes.c_longlong),
                ("triangles_below_theta", ctypes.c_longlong), ("euler_defect", ctypes.c_longlong),
                ("min_angle_deg", ctypes.c_double), ("theta", ctypes.c_double),
                ("max_segment_deviation", ctypes.c_double), ("exempted", ctypes.c_longlong),
                ("quality_violations", ctypes.c_longlong), ("goodcos2", ctypes.c_double),
                ("tie_passed", ctypes.c_longlong)]


def certify(out: CDT, inp: CDT, theta: float, goodcos2: float = 0.0) -> dict:
    """Check `out` (a refinement of `inp`) and return the certificate fields.

    ``ok`` is True when the mesh is a valid constrained Delaunay triangulation
    that preserves every input point and segment and meets the angle bound:
    every triangle with an angle below theta (decided exactly against
    goodcos2, the FP64 cos^2(theta) of the refiner's bad-triangle test; 0 = the
    host's cos()) is one the reference's equidistant-split exemption covers
    (``exempted``, GPU_Refine/refine.cu:426-493) or one the reference's FP64
    smallest-angle test passes because its two shortest edges compare equal
    and the test then measures the angle opposite edge 2 (``tie_passed``,
    refine.cu:343-358); the others are ``quality_violations``.  ``min_angle_deg``
    reports the smallest angle.
    """
    lib = _native.host()
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.gqm_certify.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ctypes.c_int, dp,
                                ctypes.c_int, ip, ctypes.c_double, ctypes.c_double, ctypes.POINTER(_Cert)]
    c = _Cert()
    rc = lib.gqm_certify(out.numberofpoints, _native.dptr(out.pointlist), out.numberoftriangles,
                         _native.iptr(out.trianglelist), _native.iptr(out.neighborlist), out.numberofsegments,
                         _native.iptr(out.segmentlist), inp.numberofpoints, _native.dptr(inp.pointlist),
                         inp.numberofsegments, _native.iptr(inp.segmentlist), float(theta), float(goodcos2),
                         ctypes.byref(c))
    d = {k: getattr(c, k) for k, _ in _Cert._fields_}
    d["ok"] = rc == 0
    return d
