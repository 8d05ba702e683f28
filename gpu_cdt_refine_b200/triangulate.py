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
        L.gqm_cdt_gpu_last_status.restype = ctypes.c_int
        L.gqm_triangulate_refine.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ctypes.POINTER(refine.Options),
                                             ctypes.POINTER(refine.CdtOut), ctypes.POINTER(refine.Stats),
                                             ctypes.POINTER(CdtGpuStats)]
        L.gqm_triangulate_refine.restype = ctypes.c_int
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
    own = _Owner(L, res)  # the arrays below view the library's memory and free it when gone
    t, s = res.numberoftriangles, res.numberofsegments
    addr = lambda p: ctypes.cast(p, ctypes.c_void_p).value  # noqa: E731
    cdt = CDT(pts.copy(), refine._view(own, addr(res.trianglelist), (t, 3), refine._I32),
              refine._view(own, addr(res.neighborlist), (t, 3), refine._I32),
              refine._view(own, addr(res.segmentlist), (s, 2), refine._I32))
    return (cdt, st.as_dict()) if with_stats else cdt


class _Owner:
    def __init__(self, L, res):
        self._L, self._res = L, res

    def __del__(self):
        try:
            self._L.gqm_cdt_gpu_free(ctypes.byref(self._res))
        except Exception:
            pass


def triangulate_refine(points: np.ndarray, segments: np.ndarray, theta=20.0, insertpolicy=refine.Offcenter,
                       mode=1, predicates=refine.PRED_REFERENCE, device=0, max_rounds=0, mlp=None,
                       max_area=0.0):
    """Points and segments in, refined mesh out, with the CDT built and refined
    on the device (no host round trip between the two).  Returns (CDT, refine
    stats, CDT-construction stats)."""
    L = _bind()
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    seg = np.ascontiguousarray(segments, dtype=np.int32).reshape(-1, 2)
    out = refine.CdtOut()
    st = refine.Stats()
    cst = CdtGpuStats()
    opt = refine.make_options(theta, insertpolicy, mode, predicates, device, max_rounds, mlp, max_area)
    rc = L.gqm_triangulate_refine(pts.shape[0], _native.dptr(pts), seg.shape[0], _native.iptr(seg),
                                  ctypes.byref(opt), ctypes.byref(out), ctypes.byref(st), ctypes.byref(cst))
    if rc == -15:
        raise CdtBuildError(L.gqm_cdt_gpu_last_status())
    if rc != 0:
        raise refine.RefineError(rc, L.gqm_status_string(rc).decode())
    return refine._take(out, False, L), st.as_dict(), cst.as_dict()


def release() -> None:
    """Frees the device buffers the builder keeps between calls."""
    _bind().gqm_cdt_gpu_release()


def main(argv=None):
    """Builds the CDT of the clustered benchmark input on the GPU and prints
    the builder's statistics (one JSON line per build); with --theta, also
    refines it in the same call (gqm_triangulate_refine) and prints both."""
    import argparse
    import json
    import time

    from . import inputs
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--points", type=int, default=2_000_000)
    p.add_argument("--segments", type=int, default=100_000)
    p.add_argument("--seed", type=int, default=20261205)
    p.add_argument("--repeat", type=int, default=1)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--theta", type=float, default=0.0, help="also refine at this angle (degrees)")
    a = p.parse_args(argv)
    pts = inputs.cluster_points(a.points, 64, 1.0e4, 5.0, 200.0, 0.10, a.seed)
    seg = inputs.pick_segments(pts, a.segments, a.seed + 1)
    for _ in range(a.repeat):
        t0 = time.perf_counter()
        if a.theta > 0:
            out, rst, st = triangulate_refine(pts, seg, theta=a.theta, device=a.device)
            st["refine"] = rst
            st["triangles"] = out.numberoftriangles
        else:
            cdt, st = build_cdt_gpu(pts, seg, device=a.device, with_stats=True)
            st["triangles"] = cdt.numberoftriangles
        st["wall_ms"] = (time.perf_counter() - t0) * 1e3
        print(json.dumps(st), flush=True)


if __name__ == "__main__":
    main()
