"""The refiner's own kernels and driver (csrc/refine.cu), compiled as host
C++ against a test-only runtime stand-in (tests/emu), agree with the oracle
byte for byte.  This checks the kernels' index arithmetic and bookkeeping on a
machine without a GPU; the GPU parity tests repeat the comparison on a B200."""
import os
import subprocess

import numpy as np
import pytest

from gpu_cdt_refine_b200 import _native, inputs, refine
from oracle import oracle_py

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "emu")
FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _emu_lib(name):
    path = os.path.join(EMU, "_build", name)
    subprocess.check_call(["make", "-s", "-C", EMU, path])
    return path


@pytest.fixture()
def emulated(request):
    saved_path, saved_lib = _native.CUDA_LIB, refine._lib
    _native.CUDA_LIB = _emu_lib(getattr(request, "param", "libgqm_emu.so"))
    refine._lib = None
    yield
    _native.CUDA_LIB, refine._lib = saved_path, saved_lib


def _same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f


@pytest.mark.parametrize("theta,policy,mode", [(20.0, 1, 1), (20.0, 1, 0), (20.0, 0, 1), (20.0, 0, 0), (15.0, 1, 1)])
def test_emulated_matches_oracle(emulated, theta, policy, mode):
    cdt = inputs.plain_small(seed=301, n=3000, nseg=200)
    got, ps, ts, st = refine.refine(cdt, theta, policy, mode, with_status=True)
    want, info = oracle_py.refine(cdt, theta, policy, mode)
    _same(got, want)
    assert np.array_equal(ps, info["pstatus"]) and np.array_equal(ts, info["tstatus"])
    assert st["rounds"] == info["rounds"]


@pytest.mark.parametrize("emulated", ["libgqm_emu_tight.so"], indirect=True)
def test_emulated_buffer_regrowth(emulated):
    """Physical buffers sized exactly to the logical capacity: every growth
    step reallocates and copies, and the result is unchanged."""
    cdt = inputs.clustered(seed=302, n=20000, nseg=1000)
    got, _ = refine.refine(cdt, 20.0, 1, 1)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    _same(got, want)


def test_emulated_round_limit(emulated):
    cdt = inputs.plain_small(seed=303, n=1000, nseg=50)
    with pytest.raises(refine.RefineError) as e:
        refine.refine(cdt, 20.0, max_rounds=1)
    assert e.value.status == -2


@pytest.mark.parametrize("field,row,col,value", [
    ("segmentlist", 0, 0, 10**6),   # segment endpoint out of range
    ("segmentlist", 1, 1, -4),      # negative endpoint
    ("trianglelist", 5, 2, 10**6),  # triangle vertex out of range
    ("neighborlist", 7, 0, 10**7),  # neighbour index out of range
])
def test_emulated_rejects_bad_indices(emulated, field, row, col, value):
    """Out-of-range indices are caught on the device before any kernel reads
    through them (GQM_ERR_ARGUMENT)."""
    cdt = inputs.plain_small(seed=304, n=500, nseg=20)
    arr = getattr(cdt, field).copy()
    arr.reshape(-1, arr.shape[-1])[row, col] = value
    setattr(cdt, field, arr)
    with pytest.raises(refine.RefineError) as e:
        refine.refine(cdt, 20.0)
    assert e.value.status == -1


def test_emulated_batch(emulated):
    doms = [inputs.plain_small(seed=310 + i, n=n, nseg=n // 20) for i, n in enumerate([300, 1500, 700])]
    got, stats = refine.refine_batch(doms, [15.0, 20.0, 18.0], workers=2)
    for d, th, g, st in zip(doms, [15.0, 20.0, 18.0], got, stats):
        want, info = oracle_py.refine(d, th, 1, 1)
        _same(g, want)
        assert st["rounds"] == info["rounds"]


def _persistent_domains():
    doms = [inputs.plain_small(seed=320 + i, n=n, nseg=max(4, n // 20)) for i, n in enumerate([300, 1500, 700, 2500])]
    doms.append(inputs.clustered(seed=329, n=2000, nseg=100))
    return doms


def test_emulated_persistent_batch_matches_oracle(emulated):
    """The persistent batch engine (csrc/batch.cu: one block refines a whole
    domain, the driver running on the device) gives each domain the oracle's
    result byte for byte, for mixed angles, modes and insertion policies."""
    doms = _persistent_domains()
    cfg = [(15.0, 1, 1), (20.0, 1, 0), (18.0, 0, 1), (20.0, 0, 0), (20.0, 1, 1)]
    for (theta, policy, mode), d in zip(cfg, doms):
        got, st = refine.refine_batch_persistent([d], theta, policy, mode)
        want, info = oracle_py.refine(d, theta, policy, mode)
        _same(got[0], want)
        assert st[0]["rounds"] == info["rounds"]
    got, st, rep = refine.refine_batch_persistent(doms, [c[0] for c in cfg], with_report=True)
    assert rep["fallbacks"] == 0
    for (theta, _, _), d, g in zip(cfg, doms, got):
        want, _ = oracle_py.refine(d, theta, 1, 1)
        _same(g, want)


def test_emulated_persistent_batch_exact_predicates(emulated):
    """Domains with exact predicates run in their own persistent launch and
    match the single-domain path with exact predicates."""
    doms = _persistent_domains()[:3]
    preds = [refine.PRED_EXACT, refine.PRED_REFERENCE, refine.PRED_EXACT]
    got, _ = refine.refine_batch_persistent(doms, 20.0, predicates=preds)
    for d, p, g in zip(doms, preds, got):
        one, _ = refine.refine(d, 20.0, predicates=p)
        _same(g, one)


@pytest.mark.parametrize("emulated", ["libgqm_emu_tight.so"], indirect=True)
def test_emulated_persistent_batch_arena_fallback(emulated):
    """Arenas with no room to grow: domains that outgrow them are refined again
    by the single-domain path, and every result is still the oracle's."""
    doms = _persistent_domains()
    got, _, rep = refine.refine_batch_persistent(doms, 20.0, with_report=True)
    assert rep["fallbacks"] > 0
    for d, g in zip(doms, got):
        want, _ = oracle_py.refine(d, 20.0, 1, 1)
        _same(g, want)


def _const_net(t):
    """A network whose output is the constant t (all weights zero)."""
    p = np.zeros(refine.MLP_PARAMS, np.float32)
    p[-1] = t
    return p


def test_emulated_learned_clamp_gives_plain(emulated):
    """Learned placement whose output is clamped (t <= 0 or t >= 1) keeps
    every off-center: the result is the plain refinement's, byte for byte."""
    cdt = inputs.plain_small(seed=331, n=2000, nseg=100)
    plain, _ = refine.refine(cdt, 20.0)
    for t in (-0.5, 1.5):
        got, st = refine.refine(cdt, 20.0, mlp=_const_net(t))
        _same(got, plain)
        assert st["learned_candidates"] > 0 and st["learned_used"] == 0


def test_emulated_learned_places_and_certifies(emulated):
    """A network answering t = 0.5 moves the candidates halfway to the
    circumcenter; the refined mesh is still a certified CDT at theta."""
    from gpu_cdt_refine_b200.certify import certify
    cdt = inputs.plain_small(seed=332, n=3000, nseg=150)
    got, st = refine.refine(cdt, 20.0, mlp=_const_net(0.5))
    assert 0 < st["learned_used"] <= st["learned_candidates"]
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert
    # the persistent batch engine applies the same rule
    gb, sb = refine.refine_batch_persistent([cdt], 20.0, mlp=_const_net(0.5))
    _same(gb[0], got)
    assert sb[0]["learned_used"] == st["learned_used"]


def test_emulated_learn_collect(emulated):
    """Training rows from a plain run: finite features, targets on the 1/8
    grid of [0, 1], one row per off-center candidate of every round."""
    cdt = inputs.plain_small(seed=333, n=2000, nseg=100)
    feat, tgt = refine.learn_collect(cdt, 20.0, cap=100000)
    _, st = refine.refine(cdt, 20.0, mlp=_const_net(-1.0))
    assert feat.shape == (st["learned_candidates"], refine.MLP_FEATURES)
    assert np.isfinite(feat).all() and np.all(feat[:, -1] == 1.0)
    assert np.all((tgt >= 0) & (tgt <= 1)) and np.allclose(tgt * 8, np.round(tgt * 8))


def test_emulated_learn_explore(emulated):
    """Exploration rows: parents precede children, drawn levels give the
    inserted t (or the off-center), the parent tree accounts for every
    inserted row and midpoint, and a seed gives the same run twice."""
    cdt = inputs.plain_small(seed=334, n=3000, nseg=150)
    r = refine.learn_explore(cdt, 20.0, levels=5, seed=7, cap=64)  # too small a cap: run again with room
    n = r["level"].shape[0]
    assert n > 64 and r["features"].shape == (n, refine.MLP_FEATURES)
    rows = np.arange(n)
    par = r["parent"]
    assert np.all((par == -1) | ((par >= 0) & (par < rows)))
    assert np.all(r["inserted"][par[par >= 0]] == 1)  # only inserted rows have descendants
    lv, tu = r["level"], r["t_used"]
    assert np.all((lv >= -1) & (lv < 5))
    assert np.all((tu == 0) | np.isclose(tu, lv / 4.0))
    assert np.all(tu[lv <= 0] == 0) and np.any(tu > 0)
    assert np.all(r["features"][lv < 0] == 0) and np.all(r["features"][lv >= 0, -1] == 1.0)
    moved = np.unique(lv[(lv > 0)])
    assert moved.size >= 3  # the draw reaches the levels
    assert np.all(r["midpoints"][r["inserted"] == 0] == 0)
    d = refine.descendants(par, r["inserted"], r["midpoints"])
    roots = (par < 0) & (r["inserted"] == 1)
    assert d[roots].sum() + roots.sum() == r["inserted"].sum() + r["midpoints"].sum()
    d1 = refine.descendants(par, r["inserted"], r["midpoints"], depth=1)
    assert np.all(d1 <= d) and np.all(d1 >= r["midpoints"])
    r2 = refine.learn_explore(cdt, 20.0, levels=5, seed=7)
    for k in r:
        assert np.array_equal(r[k], r2[k]), k
    # around a network answering t = 0.5: every candidate takes it (eps 0)
    r3 = refine.learn_explore(cdt, 20.0, levels=5, seed=7, mlp=_const_net(0.5), eps=0.0)
    cand = np.any(r3["features"] != 0, axis=1)
    assert np.all(r3["level"][cand] == -2) and np.all(r3["level"][~cand] == -1)
    assert np.all((r3["t_used"] == 0) | (r3["t_used"] == 0.5)) and np.any(r3["t_used"] == 0.5)


def test_emulated_area_bound_matches_oracle(emulated):
    """With an area bound (no counterpart in the reference; Triangle's `a`
    switch) the kernels still agree with the oracle byte for byte."""
    cdt = inputs.plain_small(seed=351, n=1500, nseg=60)
    for area in (400.0, 2000.0):
        got, st = refine.refine(cdt, 20.0, max_area=area)
        want, info = oracle_py.refine(cdt, 20.0, 1, 1, max_area=area)
        _same(got, want)
        tri = got.pointlist[got.trianglelist]
        a = 0.5 * np.abs((tri[:, 1, 0] - tri[:, 0, 0]) * (tri[:, 2, 1] - tri[:, 0, 1]) -
                         (tri[:, 1, 1] - tri[:, 0, 1]) * (tri[:, 2, 0] - tri[:, 0, 0]))
        assert a.max() <= area


def test_emulated_domain_with_hole(emulated):
    """A domain with a hole (its boundary four chains of segments) refines to
    the oracle's mesh; no triangle enters the hole."""
    from gpu_cdt_refine_b200.certify import certify
    cdt = inputs.square_with_hole(n=1500)
    got, _ = refine.refine(cdt, 20.0)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    _same(got, want)
    cen = got.pointlist[got.trianglelist].mean(axis=1)
    assert not np.any((cen[:, 0] > 0.35) & (cen[:, 0] < 0.65) & (cen[:, 1] > 0.35) & (cen[:, 1] < 0.65))
    cert = certify(got, cdt, 20.0)
    assert cert["ok"] and cert["triangles_below_theta"] == 0, cert


def test_sharded_batch_default_engine_single_rank(emulated):
    """replicas.refine_batch_sharded with its default engine (the persistent
    batch engine on this rank's device) and no process group: one rank holds
    every domain, and each result is the oracle's."""
    from gpu_cdt_refine_b200 import replicas
    doms = [inputs.plain_small(seed=67 + i, n=n, nseg=max(4, n // 25)) for i, n in enumerate((300, 500))]
    got, stats, rep = replicas.refine_batch_sharded(doms, [18.0, 20.0])
    assert rep["domains"] == [2] and len(stats) == 2
    for d, t, g in zip(doms, (18.0, 20.0), got):
        want, _ = oracle_py.refine(d, t, 1, 1)
        for f in FIELDS:
            assert np.array_equal(getattr(g, f).view(np.uint8), getattr(want, f).view(np.uint8)), f


@pytest.mark.parametrize("shape", [dict(small_cluster=8), dict(small_cluster=16, small_limit=8192),
                                   dict(small_limit=-1), dict(check_blocks_per_sm=1, step_grid=296)])
def test_emulated_launch_shapes_match_oracle(emulated, shape):
    """Every launch shape of the flip-flop loop (the one-block and cluster
    small-step kernels, grid steps only, another check-kernel budget) runs
    the same steps: the oracle's output byte for byte."""
    cdt = inputs.plain_small(seed=305, n=3000, nseg=150)
    ctx = refine.Context(0)
    try:
        ctx.set_tuning(**shape)
        assert all(ctx.tuning()[k] == v for k, v in shape.items())
        ctx.run_host(cdt, refine.make_options(20.0, 1, 1))
        got = ctx.result()
    finally:
        ctx.close()
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    _same(got, want)


def test_emulated_autotune(emulated):
    cdt = inputs.plain_small(seed=306, n=2000, nseg=100)
    ctx = refine.Context(0)
    try:
        chosen, ms = ctx.autotune(cdt, refine.make_options(20.0, 1, 1))
        assert chosen == ctx.tuning() and ms > 0
        ctx.run_host(cdt, refine.make_options(20.0, 1, 1))
        got = ctx.result()
    finally:
        ctx.close()
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    _same(got, want)
