"""Input construction: the CDT builder reproduces Triangle's "pzQnc" CDT
(the reference's input builder, GPU_Refine/mesh.cpp:397) exactly."""
import ctypes
import os

import numpy as np
import pytest

from gpu_cdt_refine_b200 import cdtio, inputs
from gpu_cdt_refine_b200.certify import certify

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TRI = os.path.join(ROOT, "oracle", "_ref", "libtriangle_ref.so")


class _TR(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int), ("nt", ctypes.c_int), ("ns", ctypes.c_int),
                ("pl", ctypes.POINTER(ctypes.c_double)), ("tl", ctypes.POINTER(ctypes.c_int)),
                ("nl", ctypes.POINTER(ctypes.c_int)), ("sl", ctypes.POINTER(ctypes.c_int)), ("ms", ctypes.c_double)]


def triangle_cdt(pts, seg):
    lib = ctypes.CDLL(TRI)
    r = _TR()
    pts = np.ascontiguousarray(pts, np.float64)
    seg = np.ascontiguousarray(seg, np.int32)
    lib.tri_ref_cdt(pts.shape[0], pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), seg.shape[0],
                    seg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(r))
    try:
        return cdtio.CDT(np.ctypeslib.as_array(r.pl, shape=(2 * r.np,)).copy(),
                         np.ctypeslib.as_array(r.tl, shape=(3 * r.nt,)).copy(),
                         np.ctypeslib.as_array(r.nl, shape=(3 * r.nt,)).copy(),
                         np.ctypeslib.as_array(r.sl, shape=(2 * r.ns,)).copy())
    finally:
        lib.tri_ref_free(ctypes.byref(r))


needs_triangle = pytest.mark.skipif(not os.path.exists(TRI), reason="reference Triangle not built")


@needs_triangle
@pytest.mark.parametrize("n,ns,seed", [(500, 20, 1), (5000, 250, 2), (20000, 1000, 3)])
def test_uniform_matches_triangle(n, ns, seed):
    pts = inputs.uniform_points(n, 0.0, 1000.0, seed)
    seg = inputs.pick_segments(pts, ns, seed + 10)
    assert seg.shape[0] == ns
    mine = inputs.build_cdt(pts, seg)
    ref = triangle_cdt(pts, seg)
    assert cdtio.same_mesh(mine, ref)


@needs_triangle
def test_clustered_matches_triangle():
    pts = inputs.cluster_points(30000, 64, 1e4, 5.0, 200.0, 0.1, 5)
    seg = inputs.pick_segments(pts, 1500, 6)
    assert cdtio.same_mesh(inputs.build_cdt(pts, seg), triangle_cdt(pts, seg))


@needs_triangle
def test_grid_circles_matches_triangle():
    c = inputs.adversarial(seed=9, g=60, nc=12, nseg=300)
    ref = triangle_cdt(c.pointlist, c.segmentlist[:300])
    assert cdtio.same_mesh(c, ref)


def test_input_is_valid_cdt():
    c = inputs.plain_small(seed=11, n=3000, nseg=150)
    cert = certify(c, c, 0.0)  # an input CDT: no angle bound
    assert cert["ok"], cert
    # convex hull enclosed by segments: no open boundary edge
    assert cert["open_boundary"] == 0


def test_segment_rules():
    pts = inputs.uniform_points(4000, 0.0, 1000.0, 21)
    seg = inputs.pick_segments(pts, 200, 22)
    ends = seg.reshape(-1)
    assert len(set(ends.tolist())) == ends.size  # endpoint-disjoint


def test_generators_deterministic():
    a = inputs.cluster_points(5000, 8, 1e3, 1.0, 20.0, 0.1, 3)
    b = inputs.cluster_points(5000, 8, 1e3, 1.0, 20.0, 0.1, 3)
    assert np.array_equal(a, b)


def test_duplicate_points_rejected():
    pts = np.array([[0, 0], [1, 0], [0, 1], [1, 0]], float)
    with pytest.raises(ValueError):
        inputs.build_cdt(pts, np.zeros((0, 2), np.int32))


def test_remove_holes_leaves_a_valid_cdt():
    """Hole removal: the triangles inside the hole are gone, every boundary
    edge is a segment, neighbours stay symmetric, and the mesh is a
    constrained Delaunay triangulation with one hole (certificate)."""
    from gpu_cdt_refine_b200.certify import certify
    c = inputs.square_with_hole(n=3000)
    cen = c.pointlist[c.trianglelist].mean(axis=1)
    assert not np.any((cen[:, 0] > 0.35) & (cen[:, 0] < 0.65) & (cen[:, 1] > 0.35) & (cen[:, 1] < 0.65))
    cert = certify(c, c, 0.0)  # an input CDT: no angle bound
    assert cert["ok"], cert
    # without holes the function returns the CDT unchanged
    d = inputs.plain_small(seed=9, n=300, nseg=10)
    assert inputs.remove_holes(d, []) is d
