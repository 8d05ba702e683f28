"""Synthetic PSLG workloads and their constrained Delaunay triangulations.

The workloads follow the five benchmark configurations of this project
(plain small, plain large clustered, adversarial structure, batched domains,
learned placement).  Points and segments come from the seeded generators in
csrc/synth.cpp and the CDT from csrc/cdt_build.cpp; everything is
deterministic for a given seed.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .cdtio import CDT


def build_cdt(points: np.ndarray, segments: np.ndarray) -> CDT:
    """CDT with the convex hull enclosed by segments (Triangle "pzQnc")."""
    lib = _native.host()
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    seg = np.ascontiguousarray(segments, dtype=np.int32).reshape(-1, 2)
    res = _native.CdtResult()
    rc = lib.gqm_cdt_build(pts.shape[0], _native.dptr(pts), seg.shape[0], _native.iptr(seg), res)
    if rc != 0:
        raise ValueError(f"CDT construction failed with status {rc}")
    try:
        t, s = res.numberoftriangles, res.numberofsegments
        tri = np.ctypeslib.as_array(res.trianglelist, shape=(t * 3,)).copy()
        nbr = np.ctypeslib.as_array(res.neighborlist, shape=(t * 3,)).copy()
        sg = np.ctypeslib.as_array(res.segmentlist, shape=(s * 2,)).copy()
    finally:
        lib.gqm_cdt_free(res)
    return CDT(pts.copy(), tri, nbr, sg)


def uniform_points(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
    xy = np.empty(2 * n, np.float64)
    m = _native.host().gqm_synth_uniform(n, lo, hi, seed, _native.dptr(xy))
    return xy[:2 * m].reshape(m, 2)


def cluster_points(n: int, k: int, L: float, smin: float, smax: float, bg: float, seed: int) -> np.ndarray:
    xy = np.empty(2 * n, np.float64)
    m = _native.host().gqm_synth_clusters(n, k, L, smin, smax, bg, seed, _native.dptr(xy))
    return xy[:2 * m].reshape(m, 2)


def pick_segments(points: np.ndarray, nseg: int, seed: int, max_gap: int = 8,
                  max_tries: int | None = None) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float64)
    out = np.empty(2 * max(nseg, 1), np.int32)
    tries = max_tries if max_tries is not None else 200 * nseg + 1000
    m = _native.host().gqm_pick_segments(pts.shape[0], _native.dptr(pts), nseg, max_gap, seed, tries,
                                         _native.iptr(out))
    return out[:2 * m].reshape(m, 2)


def filter_segments(points: np.ndarray, cand: np.ndarray, nseg: int) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float64)
    c = np.ascontiguousarray(cand, dtype=np.int32).reshape(-1, 2)
    out = np.empty(2 * max(nseg, 1), np.int32)
    m = _native.host().gqm_filter_segments(pts.shape[0], _native.dptr(pts), c.shape[0], _native.iptr(c), nseg,
                                           _native.iptr(out))
    return out[:2 * m].reshape(m, 2)


def grid_circle_points(g: int, sp: float, jit: float, nc: int, per: int, cxy: float, r0: float, r1: float,
                       seed: int):
    n = g * g + nc * per
    xy = np.empty(2 * n, np.float64)
    cid = np.empty(n, np.int32)
    m = _native.host().gqm_synth_grid_circles(g, sp, jit, nc, per, cxy, r0, r1, seed, _native.dptr(xy),
                                              _native.iptr(cid))
    return xy[:2 * m].reshape(m, 2), cid[:m]


# --- the benchmark workloads -------------------------------------------------

def plain_small(seed: int = 20261204, n: int = 10_000, nseg: int = 500) -> CDT:
    """10,000 points uniform in [0,1000]^2 with 500 random nearby-pair segments."""
    pts = uniform_points(n, 0.0, 1000.0, seed)
    seg = pick_segments(pts, nseg, seed + 1)
    return build_cdt(pts, seg)


def clustered(seed: int = 20261205, n: int = 2_000_000, nseg: int = 100_000) -> CDT:
    """64 isotropic Gaussians (centres U[0,1e4]^2, sigma log-U[5,200]) + 10% uniform."""
    pts = cluster_points(n, 64, 1.0e4, 5.0, 200.0, 0.10, seed)
    seg = pick_segments(pts, nseg, seed + 1)
    return build_cdt(pts, seg)


def adversarial(seed: int = 20261206, g: int = 700, nc: int = 200, nseg: int = 20_000,
                per: int | None = None) -> CDT:
    """Jittered g x g grid plus nc concentric circles; chords along the circles."""
    n_grid = g * g
    if per is None:
        per = max(3, n_grid // nc + (n_grid % nc > 0))  # about as many circle points as grid points
    sp = 1.0
    c = (g - 1) * sp / 2.0
    pts, cid = grid_circle_points(g, sp, 1e-9, nc, per, c, 0.05 * g * sp, 0.45 * g * sp, seed)
    cand = []
    for k in range(nc):
        idx = np.nonzero(cid == k)[0]
        ang = np.arctan2(pts[idx, 1] - c, pts[idx, 0] - c)
        idx = idx[np.argsort(ang)]
        cand.append(np.stack([idx[0:-1:2], idx[1::2]], axis=1))
    cand = np.concatenate(cand, axis=0)
    rng = np.random.default_rng(seed + 1)
    cand = cand[rng.permutation(cand.shape[0])]
    seg = filter_segments(pts, cand, nseg)
    return build_cdt(pts, seg)


def batch_domain(seed: int, nmin: int = 200, nmax: int = 50_000):
    """One domain of the batched workload: N log-uniform in [nmin, nmax],
    uniform points or a mixture of 1-8 isotropic Gaussians, segments 5% of N,
    theta drawn from {15, 18, 20} degrees.  Returns (CDT, theta)."""
    rng = np.random.default_rng(seed)
    n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
    theta = float(rng.choice([15.0, 18.0, 20.0]))
    if rng.random() < 0.5:
        pts = uniform_points(n, 0.0, 1000.0, seed)
    else:
        pts = cluster_points(n, int(rng.integers(1, 9)), 1000.0, 5.0, 100.0, 0.0, seed)
    seg = pick_segments(pts, max(1, n // 20), seed + 1)
    return build_cdt(pts, seg), theta


def batch_domains(count: int = 4096, seed: int = 20261207, nmin: int = 200, nmax: int = 50_000, threads: int = 0):
    """The batched workload: `count` independent domains (batch_domain with
    seeds seed, seed+1, ...).  The native generators release the GIL, so
    `threads` host threads build domains concurrently (0: one per core)."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    nthreads = threads or max(1, os.cpu_count() or 1)
    with ThreadPoolExecutor(nthreads) as ex:
        res = list(ex.map(lambda k: batch_domain(seed + 2 * k, nmin, nmax), range(count)))
    return [r[0] for r in res], [r[1] for r in res]


class _Mesh(ctypes.Structure):
    _fields_ = [("numberofpoints", ctypes.c_int), ("pointlist", ctypes.POINTER(ctypes.c_double)),
                ("numberoftriangles", ctypes.c_int), ("trianglelist", ctypes.POINTER(ctypes.c_int)),
                ("neighborlist", ctypes.POINTER(ctypes.c_int)), ("numberofsegments", ctypes.c_int),
                ("segmentlist", ctypes.POINTER(ctypes.c_int))]


def _mesh_args(cdt: CDT):
    p = np.ascontiguousarray(cdt.pointlist, np.float64)
    t = np.ascontiguousarray(cdt.trianglelist, np.int32)
    n = np.ascontiguousarray(cdt.neighborlist, np.int32)
    s = np.ascontiguousarray(cdt.segmentlist, np.int32)
    keep = (p, t, n, s)
    return keep, (cdt.numberofpoints, _native.dptr(p), cdt.numberoftriangles, _native.iptr(t), _native.iptr(n),
                  cdt.numberofsegments, _native.iptr(s))


def remove_holes(cdt: CDT, holes) -> CDT:
    """The CDT with every triangle reachable from a hole point without crossing
    a segment removed (Triangle's holes; the reference ignores holes), and with
    the vertices and segments that no remaining triangle uses dropped and the
    rest renumbered (gqm_remove_holes in the host library).  Hole boundaries
    must be segments; the result is a valid input of the refiner (every
    boundary edge a segment)."""
    h = np.ascontiguousarray(np.asarray(holes, np.float64).reshape(-1, 2))
    if cdt.numberoftriangles == 0 or h.shape[0] == 0:
        return cdt
    L = _native.host()
    keep, args = _mesh_args(cdt)
    m = _Mesh()
    rc = L.gqm_remove_holes(*args, h.shape[0], _native.dptr(h), ctypes.byref(m))
    if rc != 0:
        raise ValueError(f"gqm_remove_holes failed ({rc})")
    try:
        return CDT(np.ctypeslib.as_array(m.pointlist, shape=(2 * m.numberofpoints,)).copy(),
                   np.ctypeslib.as_array(m.trianglelist, shape=(3 * m.numberoftriangles,)).copy(),
                   np.ctypeslib.as_array(m.neighborlist, shape=(3 * m.numberoftriangles,)).copy(),
                   np.ctypeslib.as_array(m.segmentlist, shape=(2 * m.numberofsegments,)).copy())
    finally:
        L.gqm_mesh_free(ctypes.byref(m))


def region_attributes(cdt: CDT, regions):
    """Per-triangle (attribute, max_area) arrays from regions given as rows
    (x, y, attribute, max_area), Triangle's regionlist layout
    (gqm_region_attributes in the host library): each triangle reachable from
    a region's point without crossing a segment gets that region's values, a
    later region overwriting an earlier one; unreached triangles get 0."""
    r = np.ascontiguousarray(np.asarray(regions, np.float64).reshape(-1, 4))
    attr = np.zeros(cdt.numberoftriangles, np.float64)
    area = np.zeros(cdt.numberoftriangles, np.float64)
    keep, args = _mesh_args(cdt)
    rc = _native.host().gqm_region_attributes(*args, r.shape[0], _native.dptr(r), _native.dptr(attr),
                                              _native.dptr(area))
    if rc != 0:
        raise ValueError(f"gqm_region_attributes failed ({rc})")
    return attr, area


def square_with_hole(seed: int = 20261210, n: int = 4000, hole=(0.35, 0.65)) -> CDT:
    """A domain with a hole: n uniform points in the unit square outside the
    square hole [hole[0], hole[1]]^2, the hole's boundary as four segments
    (with points along them), the CDT built and the hole removed."""
    rng = np.random.default_rng(seed)
    lo, hi = hole
    p = rng.uniform(0.0, 1.0, (2 * n, 2))
    p = p[~((p[:, 0] > lo - 0.01) & (p[:, 0] < hi + 0.01) & (p[:, 1] > lo - 0.01) & (p[:, 1] < hi + 0.01))][:n]
    k = 16
    t = np.linspace(lo, hi, k + 1)[:-1]
    ring = np.concatenate([np.stack([t, np.full(k, lo)], 1), np.stack([np.full(k, hi), t], 1),
                           np.stack([t[::-1] + (hi - lo) / k, np.full(k, hi)], 1),
                           np.stack([np.full(k, lo), t[::-1] + (hi - lo) / k], 1)])
    pts = np.concatenate([p, ring])
    r0 = p.shape[0]
    m = ring.shape[0]
    seg = np.stack([r0 + np.arange(m), r0 + (np.arange(m) + 1) % m], 1).astype(np.int32)
    cdt = build_cdt(pts, seg)
    return remove_holes(cdt, [(0.5 * (lo + hi), 0.5 * (lo + hi))])
