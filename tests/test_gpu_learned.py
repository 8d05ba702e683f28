"""Learned Steiner placement on the B200: the network's forward and backward
kernels against the CPU restatement (oracle/mlp_oracle.py), training, and the
placement rule inside the refiner (single-domain and persistent batch)."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from gpu_cdt_refine_b200.certify import certify
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _same(a, b):
    return all(getattr(a, f).shape == getattr(b, f).shape and np.array_equal(getattr(a, f), getattr(b, f))
               for f in FIELDS)


def _rand(seed, n):
    rng = np.random.default_rng(seed)
    p = refine.mlp_init(seed, 0.3)
    p[mo.OFF_B1:mo.OFF_W2] = rng.normal(0, 0.1, 64)
    p[mo.OFF_B2:mo.OFF_W3] = rng.normal(0, 0.1, 64)
    X = rng.normal(0, 1, (n, mo.F)).astype(np.float32)
    X[:, -1] = 1.0
    T = rng.uniform(0, 1, n).astype(np.float32)
    return p, X, T


def test_infer_matches_oracle(gpu):
    # tolerance: fp32 tensor-core sums in another order than float64, and the
    # bf16 rounding of activations that may flip at a rounding boundary
    p, X, _ = _rand(1, 1000)
    y = refine.mlp_infer(p, X)
    yo = mo.forward(p, X)[3]
    assert np.max(np.abs(y - yo)) <= 2e-2 * (1 + np.max(np.abs(yo)))
    assert np.median(np.abs(y - yo)) <= 1e-3 * (1 + np.max(np.abs(yo)))


@pytest.mark.parametrize("n", [32, 100, 1000])
def test_grad_matches_oracle(gpu, n):
    p, X, T = _rand(2 + n, n)
    loss, g = refine.mlp_grad(p, X, T)
    lo, go = mo.loss_and_grad(p, X, T)
    assert abs(loss - lo) <= 1e-3 * abs(lo) + 1e-6
    assert np.linalg.norm(g - go) <= 2e-2 * np.linalg.norm(go)
    for a, b in [(mo.OFF_W1, mo.OFF_B1), (mo.OFF_W2, mo.OFF_B2), (mo.OFF_W3, mo.OFF_B3)]:
        assert np.linalg.norm(g[a:b] - go[a:b]) <= 3e-2 * np.linalg.norm(go[a:b]) + 1e-6


def test_train_fits_a_function(gpu):
    rng = np.random.default_rng(5)
    X = rng.normal(0, 1, (8192, mo.F)).astype(np.float32)
    X[:, -1] = 1.0
    T = (0.5 + 0.3 * np.tanh(X[:, 0] - 0.5 * X[:, 1])).astype(np.float32)
    p0 = refine.mlp_init(0)
    l0 = mo.loss_and_grad(p0, X, T)[0]
    p, loss = refine.mlp_train(p0, X, T, epochs=15, batch=256, lr=2e-3)
    l1 = mo.loss_and_grad(p, X, T)[0]
    assert loss < 0.2 * l0 and l1 < 0.2 * l0


def test_clamped_network_gives_plain_refinement(gpu):
    cdt = inputs.plain_small(seed=341, n=4000, nseg=200)
    plain, _ = refine.refine(cdt, 20.0)
    for t in (-1.0, 2.0):
        p = np.zeros(refine.MLP_PARAMS, np.float32)
        p[-1] = t
        got, st = refine.refine(cdt, 20.0, mlp=p)
        assert _same(got, plain) and st["learned_used"] == 0 and st["learned_candidates"] > 0


def test_constant_network_places_and_certifies(gpu):
    cdt = inputs.clustered(seed=342, n=6000, nseg=300)
    p = np.zeros(refine.MLP_PARAMS, np.float32)
    p[-1] = 0.5
    got, st = refine.refine(cdt, 20.0, mlp=p)
    assert st["learned_used"] > 0
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert
    gb, sb = refine.refine_batch_persistent([cdt, cdt], 20.0, mlp=p)
    assert _same(gb[0], got) and _same(gb[1], got)


def test_trained_network_against_plain(gpu):
    """What the trained network (gpu_cdt_refine_b200/data/placement_mlp.npy,
    trained on descendant counts of exploration runs) gains over the plain
    off-center rule on held-out inputs of the clustered distribution it was
    trained on: both meshes are certified at theta, and the learned rule
    inserts fewer vertices on every input (measured: 1.8-2.1 % fewer)."""
    import os
    p = np.load(os.path.join(os.path.dirname(refine.__file__), "data", "placement_mlp.npy")).astype(np.float32)
    gains = []
    for s in range(2):
        cdt = inputs.clustered(seed=9100 + s, n=100_000, nseg=5000)
        a, _ = refine.refine(cdt, 20.0)
        b, st = refine.refine(cdt, 20.0, mlp=p)
        for m in (a, b):
            cert = certify(m, cdt, 20.0)
            assert cert["ok"] and cert["triangles_below_theta"] == 0 and cert["min_angle_deg"] >= 20.0
        assert 0 < st["learned_used"] < st["learned_candidates"]
        gains.append((a.numberofpoints - b.numberofpoints) / a.numberofpoints)
    print(f"\nvertex reduction of the learned rule: {[f'{100 * g:.2f}%' for g in gains]}")
    assert all(g > 0.005 for g in gains)


def test_explore_rows_form_a_parent_tree(gpu):
    """Exploration run on the B200 (rows in the order the device claims
    them): parents precede children and are inserted rows, the inserted t is
    the drawn level's or the off-center, and the tree accounts for every
    inserted row and midpoint."""
    cdt = inputs.clustered(seed=9200, n=50_000, nseg=2500)
    r = refine.learn_explore(cdt, 20.0, levels=5, seed=3)
    par, ins, lv, tu = r["parent"], r["inserted"], r["level"], r["t_used"]
    n = par.shape[0]
    assert n > 0 and np.all((par == -1) | ((par >= 0) & (par < np.arange(n))))
    assert np.all(ins[par[par >= 0]] == 1)
    assert np.all((tu == 0) | np.isclose(tu, lv / 4.0)) and np.any(tu > 0)
    assert np.isfinite(r["features"]).all()
    d = refine.descendants(par, ins, r["midpoints"])
    roots = (par < 0) & (ins == 1)
    assert d[roots].sum() + roots.sum() == ins.sum() + r["midpoints"].sum()
