"""ctypes bindings of the test oracle (oracle/_build/libgqm_oracle.so, and
libgqm_oracle_fma.so: the same restatement with the products fused that the
reference as its project builds it fuses).

Test infrastructure: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libgqm_oracle.so")
LIB_FMA = os.path.join(HERE, "_build", "libgqm_oracle_fma.so")


class OracleOut(ctypes.Structure):
    _fields_ = [("numberofpoints", ctypes.c_int), ("numberoftriangles", ctypes.c_int),
                ("numberofsegments", ctypes.c_int),
                ("pointlist", ctypes.POINTER(ctypes.c_double)),
                ("trianglelist", ctypes.POINTER(ctypes.c_int)),
                ("neighborlist", ctypes.POINTER(ctypes.c_int)),
                ("segmentlist", ctypes.POINTER(ctypes.c_int)),
                ("pstatus", ctypes.POINTER(ctypes.c_ubyte)),
                ("tstatus", ctypes.POINTER(ctypes.c_ubyte)),
                ("rounds", ctypes.c_int), ("status", ctypes.c_int),
                ("flip_steps", ctypes.c_longlong), ("steiner_inserted", ctypes.c_longlong),
                ("midpoints_inserted", ctypes.c_longlong), ("bad_total", ctypes.c_longlong)]


_libs = {}


def lib(contracted=False):
    path = LIB_FMA if contracted else LIB
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.gqm_oracle_refine.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.POINTER(OracleOut)]
        L.gqm_oracle_refine.restype = ctypes.c_int
        L.gqm_oracle_refine_gc.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                           ctypes.POINTER(OracleOut)]
        L.gqm_oracle_refine_gc.restype = ctypes.c_int
        L.gqm_oracle_free.argtypes = [ctypes.POINTER(OracleOut)]
        L.gqm_oracle_set_max_area.argtypes = [ctypes.c_double]
        for f in ("gqm_oracle_orient",):
            getattr(L, f).argtypes = [dp, dp, dp]
            getattr(L, f).restype = ctypes.c_double
        for f in ("gqm_oracle_incircle", "gqm_oracle_incircle_exact"):
            getattr(L, f).argtypes = [dp, dp, dp, dp]
            getattr(L, f).restype = ctypes.c_double
        L.gqm_oracle_circumcenter.argtypes = [dp, dp, dp, ctypes.c_double, ctypes.c_int, dp]
        _libs[path] = L
    return _libs[path]


def refine(cdt, theta=20.0, policy=1, mode=1, max_rounds=100000, goodcos2=None, max_area=0.0, contracted=False):
    """Run the oracle on a CDT; returns (CDT, info dict).  goodcos2: cos^2(theta)
    as the device evaluates it (None: the host's cos()); contracted: the
    arithmetic of the reference as its project builds it (fused products)."""
    from gpu_cdt_refine_b200.cdtio import CDT
    L = lib(contracted)
    out = OracleOut()
    p = np.ascontiguousarray(cdt.pointlist, np.float64)
    t = np.ascontiguousarray(cdt.trianglelist, np.int32)
    n = np.ascontiguousarray(cdt.neighborlist, np.int32)
    s = np.ascontiguousarray(cdt.segmentlist, np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    L.gqm_oracle_set_max_area(float(max_area))
    try:
        rc = L.gqm_oracle_refine_gc(p.shape[0], p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t.shape[0],
                                    t.ctypes.data_as(ip), n.ctypes.data_as(ip), s.shape[0], s.ctypes.data_as(ip),
                                    float(theta), float(goodcos2 or 0.0), int(policy), int(mode), int(max_rounds),
                                    ctypes.byref(out))
    finally:
        L.gqm_oracle_set_max_area(0.0)
    info = dict(status=rc, rounds=out.rounds, flip_steps=out.flip_steps, steiner=out.steiner_inserted,
                midpoints=out.midpoints_inserted, bad_total=out.bad_total)
    if rc != 0:
        L.gqm_oracle_free(ctypes.byref(out))
        raise RuntimeError(f"oracle failed: {info}")
    try:
        np_, nt_, ns_ = out.numberofpoints, out.numberoftriangles, out.numberofsegments
        res = CDT(np.ctypeslib.as_array(out.pointlist, shape=(2 * np_,)).copy(),
                  np.ctypeslib.as_array(out.trianglelist, shape=(3 * nt_,)).copy(),
                  np.ctypeslib.as_array(out.neighborlist, shape=(3 * nt_,)).copy(),
                  np.ctypeslib.as_array(out.segmentlist, shape=(2 * ns_,)).copy())
        info["pstatus"] = np.ctypeslib.as_array(out.pstatus, shape=(np_,)).copy()
        info["tstatus"] = np.ctypeslib.as_array(out.tstatus, shape=(nt_,)).copy()
    finally:
        L.gqm_oracle_free(ctypes.byref(out))
    return res, info
