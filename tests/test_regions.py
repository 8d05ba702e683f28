"""Holes and regional attributes (csrc/regions.cpp, host library)."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs
from gpu_cdt_refine_b200.certify import certify
from oracle import oracle_py


def _square_with_inner_square(n=3000, seed=5, lo=0.3, hi=0.7):
    """Unit square with an inner square [lo, hi]^2 whose boundary is four
    chains of segments (the inner square is a region, not a hole)."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, (2 * n, 2))
    near = (np.abs(p[:, 0] - lo) < 0.01) | (np.abs(p[:, 0] - hi) < 0.01) | \
        (np.abs(p[:, 1] - lo) < 0.01) | (np.abs(p[:, 1] - hi) < 0.01)
    p = p[~near][:n]
    k = 12
    t = np.linspace(lo, hi, k + 1)[:-1]
    ring = np.concatenate([np.stack([t, np.full(k, lo)], 1), np.stack([np.full(k, hi), t], 1),
                           np.stack([hi + lo - t, np.full(k, hi)], 1), np.stack([np.full(k, lo), hi + lo - t], 1)])
    pts = np.concatenate([ring, p])
    m = ring.shape[0]
    seg = np.stack([np.arange(m), (np.arange(m) + 1) % m], 1).astype(np.int32)
    return inputs.build_cdt(pts, seg)


def _centroids(c):
    return c.pointlist.reshape(-1, 2)[c.trianglelist.reshape(-1, 3)].mean(axis=1)


def test_region_attributes_on_input_and_refined_mesh():
    cdt = _square_with_inner_square()
    regions = [(0.5, 0.5, 2.0, 0.01), (0.05, 0.05, 1.0, 0.0)]
    for mesh in (cdt, oracle_py.refine(cdt, 20.0, 1, 1)[0]):
        attr, area = inputs.region_attributes(mesh, regions)
        cen = _centroids(mesh)
        inside = (cen[:, 0] > 0.3) & (cen[:, 0] < 0.7) & (cen[:, 1] > 0.3) & (cen[:, 1] < 0.7)
        assert np.all(attr[inside] == 2.0) and np.all(attr[~inside] == 1.0)
        assert np.all(area[inside] == 0.01) and np.all(area[~inside] == 0.0)


def test_region_order_and_unreached():
    cdt = _square_with_inner_square()
    attr, _ = inputs.region_attributes(cdt, [(0.5, 0.5, 2.0, 0.0), (0.45, 0.55, 7.0, 0.0)])
    cen = _centroids(cdt)
    inside = (cen[:, 0] > 0.3) & (cen[:, 0] < 0.7) & (cen[:, 1] > 0.3) & (cen[:, 1] < 0.7)
    assert np.all(attr[inside] == 7.0)  # the later region overwrites
    assert np.all(attr[~inside] == 0.0)  # no region reaches the outside


def test_remove_holes_matches_centroid_test_and_refines():
    cdt = _square_with_inner_square()
    out = inputs.remove_holes(cdt, [(0.5, 0.5)])
    cen = _centroids(out)
    assert not np.any((cen[:, 0] > 0.3) & (cen[:, 0] < 0.7) & (cen[:, 1] > 0.3) & (cen[:, 1] < 0.7))
    assert out.numberoftriangles == int(np.sum(~((_centroids(cdt)[:, 0] > 0.3) & (_centroids(cdt)[:, 0] < 0.7) &
                                                  (_centroids(cdt)[:, 1] > 0.3) & (_centroids(cdt)[:, 1] < 0.7))))
    assert certify(out, out, 0.0)["ok"]
    ref, _ = oracle_py.refine(out, 20.0, 1, 1)
    cert = certify(ref, out, 20.0)
    assert cert["ok"], cert
    # a hole point outside the domain removes nothing
    same = inputs.remove_holes(cdt, [(5.0, 5.0)])
    assert same.numberoftriangles == cdt.numberoftriangles


def test_bad_indices_rejected():
    cdt = _square_with_inner_square(n=200)
    bad = inputs.CDT(cdt.pointlist, cdt.trianglelist.copy(), cdt.neighborlist, cdt.segmentlist)
    bad.trianglelist.reshape(-1)[4] = 10 ** 6
    with pytest.raises(ValueError):
        inputs.remove_holes(bad, [(0.5, 0.5)])
    with pytest.raises(ValueError):
        inputs.region_attributes(bad, [(0.5, 0.5, 1.0, 0.0)])
