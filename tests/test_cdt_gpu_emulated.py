"""GPU CDT construction (csrc/cdt_gpu.cu), compiled as host C++ against the
test-only runtime stand-in (tests/emu): the same triangulation as the exact
CPU builder and Triangle's "pzQnc" (GPU_Refine/mesh.cpp:397), the exact
certificate on degenerate inputs, and every error path.  The GPU tests repeat
the comparisons on a B200 (tests/test_gpu_cdt.py)."""
import os
import subprocess

import numpy as np
import pytest

from gpu_cdt_refine_b200 import _native, cdtio, inputs, refine, triangulate
from gpu_cdt_refine_b200.certify import certify

from test_cdt_build import needs_triangle, triangle_cdt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "emu")


@pytest.fixture(scope="module")
def emulated():
    path = os.path.join(EMU, "_build", "libgqm_emu.so")
    subprocess.check_call(["make", "-s", "-C", EMU, path])
    saved_path, saved_lib = _native.CUDA_LIB, refine._lib
    _native.CUDA_LIB = path
    refine._lib = None
    yield
    _native.CUDA_LIB, refine._lib = saved_path, saved_lib


def _valid(c, pts, seg):
    cert = certify(c, cdtio.CDT(pts, np.zeros((0, 3)), np.zeros((0, 3)), seg), 0.0)
    assert cert["ok"], cert
    assert cert["open_boundary"] == 0
    return cert


def _segset(c):
    return {tuple(sorted(s)) for s in c.segmentlist.tolist()}


@pytest.mark.parametrize("n,ns,seed", [(50, 5, 1), (300, 30, 2), (2000, 200, 3), (5000, 500, 4)])
def test_uniform_matches_cpu_builder(emulated, n, ns, seed):
    pts = inputs.uniform_points(n, 0.0, 1000.0, seed)
    seg = inputs.pick_segments(pts, ns, seed + 10)
    ref = inputs.build_cdt(pts, seg)
    g, st = triangulate.build_cdt_gpu(pts, seg, with_stats=True)
    assert cdtio.same_mesh(ref, g)
    # input segments first, in input order
    assert np.array_equal(g.segmentlist[:seg.shape[0]], seg)
    assert st["segments_missing"] > 0 or n < 100
    assert g.numberoftriangles == 2 * n - st["hull_vertices"] - 2


def test_clustered_matches_cpu_builder(emulated):
    pts = inputs.cluster_points(20000, 8, 1e4, 5.0, 200.0, 0.1, 3)
    seg = inputs.pick_segments(pts, 1000, 4)
    assert cdtio.same_mesh(inputs.build_cdt(pts, seg), triangulate.build_cdt_gpu(pts, seg))


@needs_triangle
def test_matches_triangle(emulated):
    pts = inputs.cluster_points(8000, 16, 1e3, 1.0, 30.0, 0.2, 7)
    seg = inputs.pick_segments(pts, 400, 8)
    assert cdtio.same_mesh(triangulate.build_cdt_gpu(pts, seg), triangle_cdt(pts, seg))


def test_deterministic(emulated):
    pts = inputs.uniform_points(3000, 0.0, 1.0, 12)
    seg = inputs.pick_segments(pts, 300, 13)
    a, b = triangulate.build_cdt_gpu(pts, seg), triangulate.build_cdt_gpu(pts, seg)
    for f in ("trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(a, f), getattr(b, f))


def test_grid_circles_certified(emulated):
    """Jittered grid and concentric circles (cocircular and near-collinear
    points): a valid CDT with the CPU builder's triangle and segment counts."""
    c = inputs.adversarial(seed=9, g=40, nc=8, nseg=120)
    seg = c.segmentlist[:120]
    g = triangulate.build_cdt_gpu(c.pointlist, seg)
    _valid(g, c.pointlist, seg)
    assert g.numberoftriangles == c.numberoftriangles
    assert _segset(g) == _segset(c)


def test_integer_grid_certified(emulated):
    """Exactly collinear and cocircular points everywhere; collinear hull
    points are vertices with hull segments between them."""
    xs, ys = np.meshgrid(np.arange(30.0), np.arange(20.0))
    pts = np.stack([xs.ravel(), ys.ravel()], axis=1)
    rng = np.random.default_rng(5)
    pts = pts[rng.permutation(pts.shape[0])]
    g = triangulate.build_cdt_gpu(pts, np.zeros((0, 2), np.int32))
    _valid(g, pts, np.zeros((0, 2), np.int32))
    H = 2 * (30 + 20) - 4
    assert g.numberoftriangles == 2 * pts.shape[0] - H - 2
    assert g.numberofsegments == H


@pytest.mark.parametrize("n", [3, 4, 17, 400])
def test_convex_position(emulated, n):
    """No interior point (the hull polygon is clipped instead of fanned)."""
    a = np.arange(n) * 2 * np.pi / n
    pts = np.stack([np.cos(a), np.sin(a)], axis=1) * 100.0
    g = triangulate.build_cdt_gpu(pts, np.zeros((0, 2), np.int32))
    _valid(g, pts, np.zeros((0, 2), np.int32))
    assert g.numberoftriangles == n - 2


def test_hull_with_flat_vertices_only(emulated):
    """A triangle with extra points on its edges and nothing inside."""
    pts = [[0, 0], [4, 0], [0, 4], [1, 0], [2, 0], [3, 0], [0, 1], [0, 3], [2, 2], [1, 3]]
    pts = np.array(pts, float)
    g = triangulate.build_cdt_gpu(pts, np.zeros((0, 2), np.int32))
    _valid(g, pts, np.zeros((0, 2), np.int32))
    assert g.numberoftriangles == pts.shape[0] - 2


def test_repeated_and_hull_segments(emulated):
    """A repeated segment (either direction) is kept once at its first
    occurrence; an input segment on the hull is not repeated as a hull edge."""
    pts = inputs.uniform_points(500, 0.0, 10.0, 31)
    seg = inputs.pick_segments(pts, 20, 32)
    ref0 = inputs.build_cdt(pts, np.zeros((0, 2), np.int32))
    hull_edge = ref0.segmentlist[0]
    seg2 = np.concatenate([seg, seg[3:4, ::-1], seg[5:6], hull_edge[None, :]]).astype(np.int32)
    ref = inputs.build_cdt(pts, seg2)
    g = triangulate.build_cdt_gpu(pts, seg2)
    assert cdtio.same_mesh(ref, g)
    assert np.array_equal(g.segmentlist[:21], np.concatenate([seg, hull_edge[None, :]]))
    assert g.numberofsegments == ref.numberofsegments


@pytest.mark.parametrize("case,status", [
    ("few", -1), ("collinear", -2), ("seg_index", -4), ("seg_self", -4), ("cross", -6),
    ("through", -7), ("dup_inside", -8), ("dup_hull", -8)])
def test_errors(emulated, case, status):
    rng = np.random.default_rng(3)
    pts = rng.uniform(0.0, 1.0, (200, 2))
    pts = np.concatenate([np.array([[-1.0, -1.0], [2.0, -1.0], [2.0, 2.0], [-1.0, 2.0]]), pts])
    seg = np.zeros((0, 2), np.int32)
    if case == "few":
        pts = pts[:2]
    elif case == "collinear":
        pts = np.stack([np.arange(50.0), 2.0 * np.arange(50.0)], axis=1)
    elif case == "seg_index":
        seg = np.array([[0, 999]], np.int32)
    elif case == "seg_self":
        seg = np.array([[5, 5]], np.int32)
    elif case == "cross":
        seg = np.array([[0, 2], [1, 3]], np.int32)
    elif case == "through":
        pts = np.concatenate([pts, [[0.5, 0.5]]])
        seg = np.array([[0, 2]], np.int32)  # (-1,-1)-(2,2) passes through (0.5, 0.5)
    elif case == "dup_inside":
        pts = np.concatenate([pts, pts[10:11]])
    elif case == "dup_hull":
        pts = np.concatenate([pts, pts[1:2]])
    with pytest.raises(triangulate.CdtBuildError) as e:
        triangulate.build_cdt_gpu(pts, seg)
    assert e.value.status == status
    # the builder stays usable after an error
    ok = triangulate.build_cdt_gpu(rng.uniform(0.0, 1.0, (50, 2)), np.zeros((0, 2), np.int32))
    assert ok.numberoftriangles > 0


def test_triangulate_refine_equals_two_calls(emulated):
    """The fused call (CDT built and refined on the device) gives the bytes of
    building the CDT and then refining it."""
    pts = inputs.uniform_points(3000, 0.0, 1000.0, 41)
    seg = inputs.pick_segments(pts, 150, 42)
    cdt = triangulate.build_cdt_gpu(pts, seg)
    two, _ = refine.refine(cdt, theta=20.0)
    one, st, cst = triangulate.triangulate_refine(pts, seg, theta=20.0)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(one, f), getattr(two, f)), f
    assert cst["hull_vertices"] > 2 and st["rounds"] > 0
    cert = certify(one, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert
    with pytest.raises(triangulate.CdtBuildError) as e:
        triangulate.triangulate_refine(np.concatenate([pts, pts[:1]]), seg)
    assert e.value.status == -8
