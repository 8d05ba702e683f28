"""Launch shapes of the flip-flop loop (gqm_tuning) and the autotuner.

No launch shape may change a result: the grid-wide step kernels, the
one-block small-step kernel and the thread-block-cluster small-step kernel
all make the reference's decisions (GPU_Refine/refine.cu:2328-2490), so every
shape gives the oracle's output byte for byte."""
import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from oracle import oracle_py

pytestmark = pytest.mark.gpu

FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")
SHAPES = [
    dict(),                                        # defaults
    dict(check_blocks_per_sm=1),                   # check kernel at up to 255 registers
    dict(small_limit=-1),                          # every step on the grid kernels
    dict(small_cluster=8),                         # small steps on a cluster of 8 blocks
    dict(small_cluster=16, small_limit=8192),      # ... of 16 blocks, larger steps too
    dict(step_grid=148 * 2, small_limit=512),
    dict(step_grid=148 * 8, check_blocks_per_sm=1, small_cluster=8, small_limit=4096),
]


def _same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f


@pytest.fixture(scope="module")
def cases():
    return {"cl8k": inputs.clustered(seed=203, n=8000, nseg=400),
            "u5k": inputs.plain_small(seed=202, n=5000, nseg=600),
            "cl200k": inputs.clustered(seed=404, n=200_000, nseg=10_000)}


@pytest.fixture(scope="module")
def oracle_out(cases):
    return {(k, p, m): oracle_py.refine(c, 20.0, p, m)[0] for k, c in cases.items() for p, m in ((1, 1), (0, 0))}


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()) or "default")
@pytest.mark.parametrize("case", ["cl8k", "u5k", "cl200k"])
@pytest.mark.parametrize("policy,mode", [(1, 1), (0, 0)])
def test_shape_keeps_oracle_output(gpu, cases, oracle_out, shape, case, policy, mode):
    ctx = refine.Context(0)
    try:
        ctx.set_tuning(**shape)
        opt = refine.make_options(20.0, policy, mode)
        st = ctx.run_host(cases[case], opt)
        got = ctx.result()
        t = ctx.tuning()
    finally:
        ctx.close()
    for k, v in shape.items():
        assert t[k] == v
    _same(got, oracle_out[(case, policy, mode)])
    if shape.get("small_limit", 0) < 0:
        assert st["flip_steps"] > 0


def test_exact_predicates_cluster_shape(gpu, cases):
    """The exact-predicate kernels in the cluster small-step kernel agree with
    the one-block kernel."""
    outs = []
    for shape in (dict(), dict(small_cluster=16, small_limit=8192)):
        ctx = refine.Context(0)
        try:
            ctx.set_tuning(**shape)
            ctx.run_host(cases["cl200k"], refine.make_options(20.0, 1, 1, refine.PRED_EXACT))
            outs.append(ctx.result())
        finally:
            ctx.close()
    _same(outs[0], outs[1])


def test_invalid_shapes_rejected(gpu):
    ctx = refine.Context(0)
    try:
        before = ctx.tuning()
        for bad in (dict(small_cluster=3), dict(check_blocks_per_sm=4), dict(step_grid=-5)):
            with pytest.raises(refine.RefineError):
                ctx.set_tuning(**bad)
        assert ctx.tuning() == before
    finally:
        ctx.close()


def test_autotune_picks_a_shape_and_keeps_results(gpu, cases, oracle_out):
    ctx = refine.Context(0)
    try:
        opt = refine.make_options(20.0, 1, 1)
        chosen, ms = ctx.autotune(cases["cl200k"], opt)
        assert ms > 0 and chosen == ctx.tuning()
        assert chosen["check_blocks_per_sm"] in (1, 2) and chosen["small_cluster"] in (1, 8, 16)
        ctx.run_host(cases["cl200k"], opt)
        _same(ctx.result(), oracle_out[("cl200k", 1, 1)])
    finally:
        ctx.close()
