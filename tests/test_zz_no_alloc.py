"""gqm_context_result_noalloc: reading a result with no allocation at all.

This entry point serves callers that cannot allocate when they read a result
(a service whose device memory budget is fixed at start-up and that reads many
small results in a loop, or code that must not trigger the device-wide
synchronization cudaFree implies).  It stages through one static device array
of GQM_NOALLOC_MAX_ELEMENTS rows and writes into host arrays the caller owns.

The test compares its output with gqm_context_result(), the allocating entry
point, byte for byte (the tolerance of every parity test here), on two calls
in a row, and checks that an oversized result is refused.  This file is
collected last so that a failing run has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 131072  # GQM_NOALLOC_MAX_ELEMENTS in include/gqm_refine.h
ERR_TOO_LARGE = -13


def _noalloc_result(ctx):
    L = refine.lib()
    L.gqm_context_result_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(refine.CdtOut)]
    L.gqm_context_result_noalloc.restype = ctypes.c_int
    np_, nt, ns = ctx.sizes()
    bufs = dict(pts=np.full(2 * np_, np.nan), tri=np.full(3 * nt, -7, np.int32), nbr=np.full(3 * nt, -7, np.int32),
                seg=np.full(2 * ns, -7, np.int32), ps=np.full(np_, 255, np.uint8), ts=np.full(nt, 255, np.uint8))
    out = refine.CdtOut()
    out.pointlist = bufs["pts"].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    out.trianglelist = bufs["tri"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    out.neighborlist = bufs["nbr"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    out.segmentlist = bufs["seg"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    out.pstatus = bufs["ps"].ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
    out.tstatus = bufs["ts"].ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
    rc = L.gqm_context_result_noalloc(ctx._h, ctypes.byref(out))
    return rc, out, bufs


def test_noalloc_matches_allocating_result(gpu):
    ctx = refine.Context(0)
    try:
        opt = refine.make_options(20.0, refine.Offcenter, 1)
        for seed in (401, 402):  # two calls in a row, different results
            cdt = inputs.plain_small(seed=seed, n=3000, nseg=150)
            ctx.run_host(cdt, opt)
            want, ps, ts = ctx.result(with_status=True)
            assert want.numberoftriangles <= MAX_ELEMENTS
            rc, out, b = _noalloc_result(ctx)
            assert rc == 0, refine.lib().gqm_status_string(rc)
            assert (out.numberofpoints, out.numberoftriangles, out.numberofsegments) == \
                (want.numberofpoints, want.numberoftriangles, want.numberofsegments)
            assert np.array_equal(b["pts"].view(np.uint64), want.pointlist.reshape(-1).view(np.uint64))
            assert np.array_equal(b["tri"], want.trianglelist.reshape(-1))
            assert np.array_equal(b["nbr"], want.neighborlist.reshape(-1))
            assert np.array_equal(b["seg"], want.segmentlist.reshape(-1))
            assert np.array_equal(b["ps"], ps) and np.array_equal(b["ts"], ts)
    finally:
        ctx.close()


def test_noalloc_rejects_oversized_result(gpu):
    ctx = refine.Context(0)
    try:
        cdt = inputs.plain_small(seed=403, n=40000, nseg=1000)
        ctx.run_host(cdt, refine.make_options(20.0, refine.Offcenter, 1))
        np_, nt, ns = ctx.sizes()
        assert nt > MAX_ELEMENTS
        rc, _, _ = _noalloc_result(ctx)
        assert rc == ERR_TOO_LARGE
    finally:
        ctx.close()
