"""Predicates: exact mode against rational arithmetic; reference mode against
the oracle's restatement of GPU_Refine/cudaCCW.h (zero filter constants)."""
import ctypes
from fractions import Fraction

import numpy as np
import pytest

from gpu_cdt_refine_b200 import _native
from oracle import oracle_py

DP = ctypes.POINTER(ctypes.c_double)


def _fn(name, nargs):
    f = getattr(_native.host(), name)
    f.argtypes = [DP] * nargs
    f.restype = ctypes.c_double
    return f


def _p(x):
    a = np.ascontiguousarray(x, dtype=np.float64)
    return a, a.ctypes.data_as(DP)


def orient_q(a, b, c):
    a, b, c = [tuple(map(Fraction, p)) for p in (a, b, c)]
    return (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0])


def incircle_q(a, b, c, d):
    a, b, c, d = [tuple(map(Fraction, p)) for p in (a, b, c, d)]
    adx, ady = a[0] - d[0], a[1] - d[1]
    bdx, bdy = b[0] - d[0], b[1] - d[1]
    cdx, cdy = c[0] - d[0], c[1] - d[1]
    al, bl, cl = adx * adx + ady * ady, bdx * bdx + bdy * bdy, cdx * cdx + cdy * cdy
    return al * (bdx * cdy - cdx * bdy) + bl * (cdx * ady - adx * cdy) + cl * (adx * bdy - bdx * ady)


def sign(x):
    return (x > 0) - (x < 0)


def _cases(rng, n):
    out = []
    for k in range(n):
        kind = k % 4
        if kind == 0:  # random
            pts = rng.uniform(-1e3, 1e3, size=(4, 2))
        elif kind == 1:  # nearly collinear: c on segment ab up to one ulp
            a, b = rng.uniform(-1e3, 1e3, size=(2, 2))
            t = rng.uniform(0, 1)
            c = a + t * (b - a)
            c = np.nextafter(c, c + rng.choice([-1, 1], size=2))
            pts = np.array([a, b, c, rng.uniform(-1e3, 1e3, 2)])
        elif kind == 2:  # cocircular on an integer-coordinate circle, perturbed
            r = 5.0
            base = np.array([[3.0, 4.0], [-4.0, 3.0], [-3.0, -4.0], [4.0, -3.0]]) * rng.integers(1, 1000)
            pts = base + rng.integers(-5, 5, size=2)
            if rng.uniform() < 0.5:
                pts[3] = np.nextafter(pts[3], pts[3] + 1)
        else:  # grid with tiny jitter
            pts = rng.integers(0, 4, size=(4, 2)).astype(float) + rng.choice([0.0, 1e-9, -1e-9], size=(4, 2))
        out.append(pts)
    return out


def test_orient_exact_matches_rationals():
    f = _fn("gqm_pred_orient_exact", 3)
    rng = np.random.default_rng(1)
    for pts in _cases(rng, 400):
        args = [_p(p) for p in pts[:3]]
        got = f(*[x[1] for x in args])
        assert sign(got) == sign(orient_q(*pts[:3]))


def test_incircle_exact_matches_rationals():
    f = _fn("gqm_pred_incircle_exact", 4)
    rng = np.random.default_rng(2)
    for pts in _cases(rng, 400):
        args = [_p(p) for p in pts]
        got = f(*[x[1] for x in args])
        assert sign(got) == sign(incircle_q(*pts))


def test_exact_incircle_degenerate_zero():
    f = _fn("gqm_pred_incircle_exact", 4)
    pts = [np.array(p, float) for p in ([3.0, 4.0], [-4.0, 3.0], [-3.0, -4.0], [4.0, -3.0])]
    assert f(*[_p(p)[1] for p in pts]) == 0.0


def test_reference_orient_is_plain_determinant():
    f = _fn("gqm_pred_orient_ref", 3)
    L = oracle_py.lib()
    rng = np.random.default_rng(3)
    for pts in _cases(rng, 200):
        args = [_p(p)[1] for p in pts[:3]]
        assert f(*args) == L.gqm_oracle_orient(*args)


def test_reference_zero_fallback_matches_oracle():
    """The expansion evaluated with the reference's zero splitter is the same
    sequence of operations in the product header and in the oracle."""
    f = _fn("gqm_pred_incircle_ref_fallback", 4)
    L = oracle_py.lib()
    rng = np.random.default_rng(4)
    for pts in _cases(rng, 200):
        args = [_p(p)[1] for p in pts]
        a = f(*args)
        b = L.gqm_oracle_incircle_exact(*args)
        assert np.float64(a).tobytes() == np.float64(b).tobytes()
