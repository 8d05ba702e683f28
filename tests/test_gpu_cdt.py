"""GPU CDT construction on a B200: the same triangulation as the exact CPU
builder (itself checked against Triangle's "pzQnc", GPU_Refine/mesh.cpp:397)
at the benchmark sizes, the exact certificate on degenerate inputs, error
statuses, and the refiner run on a GPU-built input."""
import time

import numpy as np
import pytest

from gpu_cdt_refine_b200 import cdtio, inputs, refine, triangulate
from gpu_cdt_refine_b200.certify import certify

pytestmark = pytest.mark.gpu


def _valid(c, pts, seg):
    cert = certify(c, cdtio.CDT(pts, np.zeros((0, 3)), np.zeros((0, 3)), seg), 0.0)
    assert cert["ok"], cert
    assert cert["open_boundary"] == 0


def _both(pts, seg):
    t0 = time.perf_counter()
    ref = inputs.build_cdt(pts, seg)
    t1 = time.perf_counter()
    triangulate.build_cdt_gpu(pts, seg)  # warm-up: allocation and module load
    t2 = time.perf_counter()
    g, st = triangulate.build_cdt_gpu(pts, seg, with_stats=True)
    t3 = time.perf_counter()
    return ref, g, st, (t1 - t0) * 1e3, (t3 - t2) * 1e3


@pytest.mark.parametrize("n,ns,seed", [(1000, 50, 1), (200_000, 10_000, 2)])
def test_uniform_matches_cpu_builder(n, ns, seed):
    pts = inputs.uniform_points(n, 0.0, 1000.0, seed)
    seg = inputs.pick_segments(pts, ns, seed + 10)
    ref, g, st, cpu_ms, gpu_ms = _both(pts, seg)
    assert cdtio.same_mesh(ref, g)
    assert np.array_equal(g.segmentlist[:seg.shape[0]], seg)
    print(f"\nuniform {n}: CPU builder {cpu_ms:.1f} ms, GPU builder {gpu_ms:.1f} ms; {st}")


def test_clustered_2m_matches_cpu_builder():
    """The benchmark input: 2,000,000 clustered points, 100,000 segments."""
    pts = inputs.cluster_points(2_000_000, 64, 1.0e4, 5.0, 200.0, 0.10, 20261205)
    seg = inputs.pick_segments(pts, 100_000, 20261206)
    ref, g, st, cpu_ms, gpu_ms = _both(pts, seg)
    assert cdtio.same_mesh(ref, g)
    print(f"\nclustered 2M: CPU builder {cpu_ms:.1f} ms, GPU builder {gpu_ms:.1f} ms (x{cpu_ms / gpu_ms:.1f}); {st}")
    assert gpu_ms < cpu_ms


def test_grid_circles_certified():
    """Jittered grid plus concentric circles with chord segments (cocircular
    and nearly collinear points)."""
    c = inputs.adversarial(seed=20261206, g=200, nc=40, nseg=4000)
    seg = c.segmentlist[:4000]
    g = triangulate.build_cdt_gpu(c.pointlist, seg)
    _valid(g, c.pointlist, seg)
    assert g.numberoftriangles == c.numberoftriangles
    assert {tuple(sorted(s)) for s in g.segmentlist.tolist()} == {tuple(sorted(s)) for s in c.segmentlist.tolist()}


def test_integer_grid_and_convex_position():
    xs, ys = np.meshgrid(np.arange(300.0), np.arange(200.0))
    pts = np.stack([xs.ravel(), ys.ravel()], axis=1)
    pts = pts[np.random.default_rng(5).permutation(pts.shape[0])]
    g = triangulate.build_cdt_gpu(pts, np.zeros((0, 2), np.int32))
    _valid(g, pts, np.zeros((0, 2), np.int32))
    assert g.numberoftriangles == 2 * pts.shape[0] - (2 * (300 + 200) - 4) - 2
    a = np.arange(1000) * 2 * np.pi / 1000
    circ = np.stack([np.cos(a), np.sin(a)], axis=1)
    g = triangulate.build_cdt_gpu(circ, np.zeros((0, 2), np.int32))
    _valid(g, circ, np.zeros((0, 2), np.int32))


@pytest.mark.parametrize("case,status", [("cross", -6), ("through", -7), ("dup_inside", -8)])
def test_errors(case, status):
    rng = np.random.default_rng(3)
    pts = np.concatenate([np.array([[-1.0, -1.0], [2.0, -1.0], [2.0, 2.0], [-1.0, 2.0]]),
                          rng.uniform(0.0, 1.0, (20000, 2))])
    seg = np.zeros((0, 2), np.int32)
    if case == "cross":
        seg = np.array([[0, 2], [1, 3]], np.int32)
    elif case == "through":
        pts = np.concatenate([pts, [[0.5, 0.5]]])
        seg = np.array([[0, 2]], np.int32)
    else:
        pts = np.concatenate([pts, pts[100:101]])
    with pytest.raises(triangulate.CdtBuildError) as e:
        triangulate.build_cdt_gpu(pts, seg)
    assert e.value.status == status
    ok = triangulate.build_cdt_gpu(pts[:1000], np.zeros((0, 2), np.int32))
    assert ok.numberoftriangles > 0


def test_refine_a_gpu_built_input():
    pts = inputs.cluster_points(100_000, 16, 1e4, 5.0, 200.0, 0.1, 77)
    seg = inputs.pick_segments(pts, 5_000, 78)
    cdt = triangulate.build_cdt_gpu(pts, seg)
    out, _ = refine.refine(cdt, theta=20.0)
    cert = certify(out, cdt, 20.0)
    assert cert["ok"], cert
    assert cert["triangles_below_theta"] <= 1


def test_triangulate_refine_2m():
    """Points and segments to refined mesh on the device: the same bytes as
    the two calls, and the time of the whole flow against the CPU builder
    followed by the refiner."""
    pts = inputs.cluster_points(2_000_000, 64, 1.0e4, 5.0, 200.0, 0.10, 20261205)
    seg = inputs.pick_segments(pts, 100_000, 20261206)
    triangulate.triangulate_refine(pts, seg)  # warm-up
    t0 = time.perf_counter()
    one, st, cst = triangulate.triangulate_refine(pts, seg)
    t1 = time.perf_counter()
    cdt = inputs.build_cdt(pts, seg)
    two, _ = refine.refine(cdt, theta=20.0)
    t2 = time.perf_counter()
    same = cdtio.same_mesh(cdt, triangulate.build_cdt_gpu(pts, seg))
    print(f"\npoints to refined mesh, 2M: fused GPU call {(t1 - t0) * 1e3:.1f} ms, CPU builder + refiner "
          f"{(t2 - t1) * 1e3:.1f} ms; CDT {cst['ms_total']:.1f} ms, output triangles {one.numberoftriangles}")
    assert same
    ref_cdt = triangulate.build_cdt_gpu(pts, seg)
    three, _ = refine.refine(ref_cdt, theta=20.0)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(one, f), getattr(three, f)), f
    assert abs(one.numberoftriangles - two.numberoftriangles) < 0.005 * two.numberoftriangles
