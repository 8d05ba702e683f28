"""Allocation failure, injected on the host: the refiner's own driver
(csrc/refine.cu compiled against the test-only runtime stand-in of tests/emu)
is made to fail each of its device and pinned allocations in turn.  Every
such call must end with GQM_ERR_MEMORY and hand out no result, and the same
context must then refine the input again exactly as the oracle does."""
import ctypes

import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine
from oracle import oracle_py

from test_emulated_kernels import FIELDS, emulated  # noqa: F401  (fixture)

ERR_MEMORY = -12


def _run(ctx, cdt, opt):
    """gqm_context_run + gqm_context_result; (status, CDT or None)."""
    L = refine.lib()
    keep = []
    cin = refine._cdt_in(cdt, keep)
    rc = L.gqm_context_run(ctx, ctypes.byref(cin), 0, ctypes.byref(opt), None)
    if rc:
        return rc, None
    out = refine.CdtOut()
    rc = L.gqm_context_result(ctx, ctypes.byref(out))
    if rc:
        assert not out.pointlist and not out.trianglelist
        return rc, None
    return 0, refine._take(out, L=L)


def test_every_allocation_failure_is_reported_and_recoverable(emulated):  # noqa: F811
    L = refine.lib()
    L.gqm_fake_fail_alloc_at.argtypes = [ctypes.c_longlong]
    L.gqm_fake_alloc_count.restype = ctypes.c_longlong
    cdt = inputs.plain_small(seed=61, n=600, nseg=30)
    want, _ = oracle_py.refine(cdt, 20.0, 1, 1)
    opt = refine.make_options(20.0, refine.Offcenter, 1)

    # allocations of one context's first refinement and result
    L.gqm_fake_fail_alloc_at(-1)
    ctx = ctypes.c_void_p()
    assert L.gqm_context_create(0, ctypes.byref(ctx)) == 0
    rc, got = _run(ctx, cdt, opt)
    assert rc == 0
    total = L.gqm_fake_alloc_count()
    L.gqm_context_destroy(ctx)
    assert total > 5

    for k in range(total):
        L.gqm_fake_fail_alloc_at(k)
        ctx = ctypes.c_void_p()
        rc = L.gqm_context_create(0, ctypes.byref(ctx))
        if rc:
            assert rc == ERR_MEMORY and not ctx.value, k
            continue
        rc, got = _run(ctx, cdt, opt)
        assert rc == ERR_MEMORY and got is None, (k, rc)
        L.gqm_fake_fail_alloc_at(-1)
        rc, got = _run(ctx, cdt, opt)  # the same context recovers
        assert rc == 0, (k, rc)
        for f in FIELDS:
            assert np.array_equal(getattr(got, f).view(np.uint8), getattr(want, f).view(np.uint8)), (k, f)
        L.gqm_context_destroy(ctx)
    L.gqm_fake_fail_alloc_at(-1)


def test_allocation_failure_while_growing_a_used_context(emulated):  # noqa: F811
    """A context that has refined a small input grows its buffers for a larger
    one; each allocation of that growth fails in turn, and the context still
    refines both inputs exactly as the oracle does afterwards."""
    L = refine.lib()
    L.gqm_fake_fail_alloc_at.argtypes = [ctypes.c_longlong]
    L.gqm_fake_alloc_count.restype = ctypes.c_longlong
    small = inputs.plain_small(seed=62, n=300, nseg=12)
    large = inputs.clustered(seed=63, n=2500, nseg=120)
    want_small, _ = oracle_py.refine(small, 20.0, 1, 1)
    want_large, _ = oracle_py.refine(large, 20.0, 1, 1)
    opt = refine.make_options(20.0, refine.Offcenter, 1)

    def fresh():
        L.gqm_fake_fail_alloc_at(-1)
        ctx = ctypes.c_void_p()
        assert L.gqm_context_create(0, ctypes.byref(ctx)) == 0
        assert _run(ctx, small, opt)[0] == 0
        return ctx

    ctx = fresh()
    L.gqm_fake_fail_alloc_at(-1)
    assert _run(ctx, large, opt)[0] == 0
    growth = L.gqm_fake_alloc_count()
    L.gqm_context_destroy(ctx)
    assert growth > 5
    for k in range(growth):
        ctx = fresh()
        L.gqm_fake_fail_alloc_at(k)
        rc, got = _run(ctx, large, opt)
        assert rc == ERR_MEMORY and got is None, (k, rc)
        L.gqm_fake_fail_alloc_at(-1)
        for cdt, want in ((large, want_large), (small, want_small)):
            rc, got = _run(ctx, cdt, opt)
            assert rc == 0, (k, rc)
            for f in FIELDS:
                assert np.array_equal(getattr(got, f).view(np.uint8), getattr(want, f).view(np.uint8)), (k, f)
        L.gqm_context_destroy(ctx)
    L.gqm_fake_fail_alloc_at(-1)


def test_allocation_failure_in_the_persistent_batch(emulated):  # noqa: F811
    """The persistent batch engine's per-device buffers (input, output, arenas,
    pinned staging, job table) are released and each of their allocations
    fails in turn: the call reports GQM_ERR_MEMORY, and the next call gives
    every domain the oracle's result."""
    L = refine.lib()
    L.gqm_fake_fail_alloc_at.argtypes = [ctypes.c_longlong]
    L.gqm_fake_alloc_count.restype = ctypes.c_longlong
    doms = [inputs.plain_small(seed=64 + i, n=n, nseg=max(4, n // 25)) for i, n in enumerate((250, 700, 400))]
    want = [oracle_py.refine(d, 20.0, 1, 1)[0] for d in doms]
    L.gqm_batch_release(0)
    L.gqm_fake_fail_alloc_at(-1)
    refine.refine_batch_persistent(doms, 20.0)
    total = L.gqm_fake_alloc_count()
    assert total >= 4
    for k in range(total):
        L.gqm_batch_release(0)
        L.gqm_fake_fail_alloc_at(k)
        with pytest.raises(refine.RefineError) as e:
            refine.refine_batch_persistent(doms, 20.0)
        assert e.value.status == ERR_MEMORY, (k, e.value.status)
        L.gqm_fake_fail_alloc_at(-1)
        got, _ = refine.refine_batch_persistent(doms, 20.0)
        for g, w in zip(got, want):
            for f in FIELDS:
                assert np.array_equal(getattr(g, f).view(np.uint8), getattr(w, f).view(np.uint8)), (k, f)
    L.gqm_batch_release(0)


def test_allocation_failure_in_the_cdt_builder(emulated):  # noqa: F811
    """The GPU CDT builder's buffers are released and each of its allocations
    fails in turn (first build, then the growth for a larger input): the call
    reports GQM_CDT_ERR_MEMORY, and the next call builds the same mesh as
    before."""
    from gpu_cdt_refine_b200 import cdtio, triangulate
    L = refine.lib()
    L.gqm_fake_fail_alloc_at.argtypes = [ctypes.c_longlong]
    L.gqm_fake_alloc_count.restype = ctypes.c_longlong
    cdt_err_memory = -11
    cases = []
    for seed, n in ((65, 400), (66, 1500)):
        pts = inputs.uniform_points(n, 0.0, 1000.0, seed)
        seg = inputs.pick_segments(pts, n // 25, seed + 1)
        cases.append((pts, seg, inputs.build_cdt(pts, seg)))

    def build(i):
        pts, seg, _ = cases[i]
        return triangulate.build_cdt_gpu(pts, seg)

    for grow in (False, True):
        triangulate._bind().gqm_cdt_gpu_release()
        if grow:
            L.gqm_fake_fail_alloc_at(-1)
            build(0)
        L.gqm_fake_fail_alloc_at(-1)
        build(1)
        total = L.gqm_fake_alloc_count()
        assert total >= 3
        for k in range(total):
            triangulate._bind().gqm_cdt_gpu_release()
            if grow:
                L.gqm_fake_fail_alloc_at(-1)
                build(0)
            L.gqm_fake_fail_alloc_at(k)
            with pytest.raises(triangulate.CdtBuildError) as e:
                build(1)
            assert e.value.status == cdt_err_memory, (grow, k, e.value.status)
            L.gqm_fake_fail_alloc_at(-1)
            for i in (0, 1):  # the smaller input first: it must not reuse a buffer that was not reallocated
                assert cdtio.same_mesh(build(i), cases[i][2]), (grow, k, i)
    triangulate._bind().gqm_cdt_gpu_release()
    L.gqm_fake_fail_alloc_at(-1)

