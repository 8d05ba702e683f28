"""The exact certificate's angle bound and the reference's exemption rule
(csrc/certify.cpp), on CPU with oracle outputs."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs
from gpu_cdt_refine_b200.certify import certify
from oracle import oracle_py


def _wedge(angle_deg):
    """Two input segments meeting at the origin at `angle_deg`, in a box."""
    a = np.radians(angle_deg)
    pts = np.array([[0.0, 0.0], [100.0, 0.0], [100 * np.cos(a), 100 * np.sin(a)], [-50.0, -50.0], [150.0, -50.0],
                    [150.0, 150.0], [-50.0, 150.0]])
    return inputs.build_cdt(pts, np.array([[0, 1], [0, 2]], dtype=np.int32))


@pytest.mark.parametrize("angle", [5.0, 10.0, 15.0])
def test_small_input_angle_is_exempted(angle):
    """Refinement cannot remove the input angle itself: the triangles that keep
    it are below theta, and each is one the reference's exemption
    (GPU_Refine/refine.cu:426-493) covers, checked by code."""
    cdt = _wedge(angle)
    out, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    cert = certify(out, cdt, 20.0)
    assert cert["triangles_below_theta"] > 0
    assert cert["exempted"] == cert["triangles_below_theta"] and cert["quality_violations"] == 0
    assert cert["ok"], cert
    assert cert["min_angle_deg"] == pytest.approx(angle, abs=1e-9)


def test_unexempted_small_angle_fails():
    """A split point moved along its segment (planted in the oracle's output):
    the two split points next to the small input angle are no longer at equal
    distance from its vertex, so the triangle between them is a violation."""
    cdt = _wedge(10.0)
    out, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    assert certify(out, cdt, 20.0)["quality_violations"] == 0
    p = out.pointlist.reshape(-1, 2)
    # the split point on the segment (0 -> 1) nearest the origin
    on_x = [i for i in range(cdt.numberofpoints, p.shape[0]) if p[i, 1] == 0.0 and 0.0 < p[i, 0] < 100.0]
    k = min(on_x, key=lambda i: p[i, 0])
    p[k, 0] *= 1.05
    cert = certify(out, cdt, 20.0)
    assert cert["quality_violations"] >= 1 and not cert["ok"]


def test_input_cdt_is_not_quality():
    """An unrefined CDT has triangles below 20 degrees that no exemption
    covers; with no angle bound (theta 0) the same mesh certifies."""
    c = inputs.plain_small(seed=11, n=3000, nseg=150)
    cert = certify(c, c, 20.0)
    assert cert["quality_violations"] == cert["triangles_below_theta"] > 0 and not cert["ok"]
    assert certify(c, c, 0.0)["ok"]


def test_angle_test_is_exact_at_the_threshold():
    """A triangle whose smallest angle is theta up to rounding: the decision
    follows the exact sign of dot^2 - c2 |u|^2 |w|^2 for the given c2, so
    nudging c2 by one unit in the last place flips it."""
    from gpu_cdt_refine_b200.cdtio import CDT
    pts = np.array([[0.0, 0.0], [4.0, 0.0], [4.0, 3.0]])  # angle at the origin: cos^2 = 16/25
    tri = CDT(pts.reshape(-1), np.array([0, 1, 2], np.int32), np.array([-1, -1, -1], np.int32),
              np.array([0, 1, 1, 2, 2, 0], np.int32))
    c2 = 16.0 / 25.0  # rounded: 0.64 is not a binary fraction
    exact = 16 * 2 ** 53 - 25 * round(c2 * 2 ** 53)  # sign of 16/25 - c2, in units of 2^-53 / 25
    below = certify(tri, tri, 36.0, goodcos2=c2)["triangles_below_theta"]
    assert below == (1 if exact > 0 else 0)
    assert certify(tri, tri, 36.0, goodcos2=np.nextafter(c2, 0.0))["triangles_below_theta"] == 1
    assert certify(tri, tri, 36.0, goodcos2=np.nextafter(c2, 1.0))["triangles_below_theta"] == 0


def _one_triangle(order):
    """One flat isosceles triangle (base (0,0)-(2,0), top (1, 0.25): base
    angles 14.04 degrees, legs of exactly equal FP64 length), all three edges
    input segments, with its vertices listed starting at `order`."""
    from gpu_cdt_refine_b200.cdtio import CDT
    pts = np.array([[0.0, 0.0], [2.0, 0.0], [1.0, 0.25]])
    tri = np.roll(np.array([0, 1, 2], dtype=np.int32), -order).reshape(1, 3)
    return CDT(pointlist=pts, trianglelist=tri, neighborlist=np.full((1, 3), -1, dtype=np.int32),
               segmentlist=np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32))


@pytest.mark.parametrize("order,passes", [(0, True), (1, False), (2, False)])
def test_length_tie_of_the_reference_test(order, passes):
    """The reference's smallest-angle routine (GPU_Refine/refine.cu:317-374)
    takes edge 2 whenever its strict comparisons of edges 0 and 1 tie.  Listed
    as (0,0), (2,0), (1,0.25) the two equal legs are edges 0 and 1: edge 2 is
    the base and the angle measured is the 152-degree top angle, so the
    reference's test passes the triangle (tie_passed).  In the other two
    vertex orders edge 2 is one of the legs and the test measures a 14-degree
    base angle: a quality violation."""
    c = _one_triangle(order)
    cert = certify(c, c, 20.0)
    assert cert["triangles_below_theta"] == 1 and cert["exempted"] == 0
    assert cert["tie_passed"] == (1 if passes else 0)
    assert cert["quality_violations"] == (0 if passes else 1)
    assert cert["ok"] == passes
    assert cert["min_angle_deg"] == pytest.approx(np.degrees(np.arctan(0.25)), abs=1e-9)
