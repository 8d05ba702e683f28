"""The CPU restatement of the placement network (oracle/mlp_oracle.py): its
backward pass is the derivative of its forward pass (finite differences in
float64), and its bf16 rounding matches the bit-level rule of the device code."""
import numpy as np

from oracle import mlp_oracle as mo


def _data(seed, n=40):
    rng = np.random.default_rng(seed)
    p = np.zeros(mo.NPARAM, np.float32)
    p[:] = rng.normal(0, 0.2, mo.NPARAM)
    X = rng.normal(0, 1, (n, mo.F)).astype(np.float32)
    T = rng.uniform(0, 1, n).astype(np.float32)
    return p.astype(np.float64), X, T


def test_backward_is_derivative_of_forward():
    p, X, T = _data(1)
    with mo.exact_arithmetic():
        _, g = mo.loss_and_grad(p, X, T)
        rng = np.random.default_rng(2)
        for i in rng.choice(mo.NPARAM, 60, replace=False):
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            num = (mo.loss_and_grad(pp, X, T)[0] - mo.loss_and_grad(pm, X, T)[0]) / (2 * h)
            assert abs(num - g[i]) <= 1e-5 + 1e-4 * abs(g[i]), (i, num, g[i])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 65504.0, 1e-20], np.float32)
    r = mo.bf16(vals)
    for v, b in zip(vals, r):
        bits = np.float32(b).view(np.uint32)
        assert bits & 0xFFFF == 0
        # nearest of the two neighbouring bf16 values
        lo = np.uint32(np.float32(v).view(np.uint32) & 0xFFFF0000).view(np.float32)
        hi = np.uint32((np.float32(v).view(np.uint32) & 0xFFFF0000) + 0x10000).view(np.float32)
        assert abs(b - v) <= min(abs(lo - v), abs(hi - v)) + 0.0
