"""ctypes bindings of the reference's vendored Triangle 1.6 (oracle/_ref).

Test and baseline infrastructure: the CDT call reproduces the reference's
input construction (triangulate("pzQnc"), GPU_Refine/mesh.cpp:397) and the
quality call its CPU refinement (triangulate("pzDQnrq<theta>") / "pzQnrq<theta>",
GPU_Refine/main.cpp:389-407).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libtriangle_ref.so")


class TriResult(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int), ("nt", ctypes.c_int), ("ns", ctypes.c_int),
                ("pl", ctypes.POINTER(ctypes.c_double)), ("tl", ctypes.POINTER(ctypes.c_int)),
                ("nl", ctypes.POINTER(ctypes.c_int)), ("sl", ctypes.POINTER(ctypes.c_int)), ("ms", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} missing: build it with `make -C oracle ref` where the reference is present")
        _lib = ctypes.CDLL(LIB)
    return _lib


def _take(r):
    from gpu_cdt_refine_b200.cdtio import CDT
    return CDT(np.ctypeslib.as_array(r.pl, shape=(2 * r.np,)).copy(),
               np.ctypeslib.as_array(r.tl, shape=(3 * r.nt,)).copy(),
               np.ctypeslib.as_array(r.nl, shape=(3 * r.nt,)).copy(),
               np.ctypeslib.as_array(r.sl, shape=(2 * r.ns,)).copy())


def cdt(points, segments, with_ms=False):
    """Triangle "pzQnc" CDT; with_ms also returns the time of the triangulate() call."""
    L = lib()
    r = TriResult()
    p = np.ascontiguousarray(points, np.float64)
    s = np.ascontiguousarray(segments, np.int32)
    L.tri_ref_cdt(p.shape[0], p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), s.shape[0],
                  s.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(r))
    try:
        return (_take(r), r.ms) if with_ms else _take(r)
    finally:
        L.tri_ref_free(ctypes.byref(r))


def quality(c, theta=20.0, mode=1, keep=False):
    """Triangle's quality refinement of CDT `c`; returns (ms, output triangles[, CDT])."""
    L = lib()
    r = TriResult()
    p = np.ascontiguousarray(c.pointlist, np.float64)
    t = np.ascontiguousarray(c.trianglelist, np.int32)
    n = np.ascontiguousarray(c.neighborlist, np.int32)
    s = np.ascontiguousarray(c.segmentlist, np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    L.tri_ref_quality.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ip, ip, ctypes.c_int,
                                  ip, ctypes.c_double, ctypes.c_int, ctypes.POINTER(TriResult)]
    L.tri_ref_quality(p.shape[0], p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t.shape[0], t.ctypes.data_as(ip),
                      n.ctypes.data_as(ip), s.shape[0], s.ctypes.data_as(ip), float(theta), int(mode), ctypes.byref(r))
    try:
        out = _take(r) if keep else None
        ms, nt = r.ms, r.nt
    finally:
        L.tri_ref_free(ctypes.byref(r))
    return (ms, nt, out) if keep else (ms, nt)
