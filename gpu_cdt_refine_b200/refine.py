"""Python host side of the refiner, mirroring the reference's interface.

``GPU_Refine_Quality(input, theta, insertpolicy, deletepolicy, mode,
debug_iter)`` has the argument meaning of GPU_Refine/refine.h:385-386 and
returns the refined CDT (plus the PStatus / TStatus debug bytes when asked).
It calls the sm_100a library through the C ABI of include/gqm_refine.h; there
is no CPU fallback: without the library or a GPU it raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native
from .cdtio import CDT

Circumcenter, Offcenter = 0, 1
Strict, Connected, Orthogonal, noDeletion, DeleteFromDT, noPriority = range(6)
PRED_REFERENCE, PRED_EXACT = 0, 1


class CdtIn(ctypes.Structure):
    _fields_ = [("numberofpoints", ctypes.c_int), ("pointlist", ctypes.c_void_p),
                ("numberoftriangles", ctypes.c_int), ("trianglelist", ctypes.c_void_p),
                ("neighborlist", ctypes.c_void_p), ("numberofsegments", ctypes.c_int),
                ("segmentlist", ctypes.c_void_p)]


class CdtOut(ctypes.Structure):
    _fields_ = [("numberofpoints", ctypes.c_int), ("pointlist", ctypes.POINTER(ctypes.c_double)),
                ("numberoftriangles", ctypes.c_int), ("trianglelist", ctypes.POINTER(ctypes.c_int)),
                ("neighborlist", ctypes.POINTER(ctypes.c_int)), ("numberofsegments", ctypes.c_int),
                ("segmentlist", ctypes.POINTER(ctypes.c_int)), ("pstatus", ctypes.POINTER(ctypes.c_ubyte)),
                ("tstatus", ctypes.POINTER(ctypes.c_ubyte))]


# the same structure with its pointers read as plain addresses (ints)
class _CdtOutAddr(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p if issubclass(t, ctypes._Pointer) else t) for n, t in CdtOut._fields_]


class Options(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_double), ("insert_policy", ctypes.c_int), ("mode", ctypes.c_int),
                ("predicates", ctypes.c_int), ("device", ctypes.c_int), ("max_rounds", ctypes.c_longlong),
                ("placement", ctypes.c_int), ("mlp", ctypes.c_void_p), ("max_area", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int), ("flip_steps", ctypes.c_longlong),
                ("steiner_inserted", ctypes.c_longlong), ("midpoints_inserted", ctypes.c_longlong),
                ("bad_total", ctypes.c_longlong), ("host_syncs", ctypes.c_longlong),
                ("kernel_launches", ctypes.c_longlong), ("exact_fallbacks", ctypes.c_longlong),
                ("goodcos2", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("learned_candidates", ctypes.c_longlong), ("learned_used", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Probe(ctypes.Structure):
    _fields_ = [("check_launches", ctypes.c_longlong), ("check_items", ctypes.c_longlong),
                ("check_ms", ctypes.c_double), ("loop_launches", ctypes.c_longlong), ("loop_ms", ctypes.c_double),
                ("first_items", ctypes.c_longlong * 4), ("small_launches", ctypes.c_longlong),
                ("small_items", ctypes.c_longlong), ("small_winners", ctypes.c_longlong), ("small_ms", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "first_items"}
        d["first_items"] = list(self.first_items)
        return d


class BatchOptions(ctypes.Structure):
    _fields_ = [("threads_per_block", ctypes.c_int), ("blocks_per_sm", ctypes.c_int),
                ("memory_fraction", ctypes.c_double)]


class BatchReport(ctypes.Structure):
    _fields_ = [("grid", ctypes.c_int), ("threads_per_block", ctypes.c_int), ("blocks_per_sm", ctypes.c_int),
                ("fallbacks", ctypes.c_int), ("arena_bytes", ctypes.c_longlong), ("kernel_ms", ctypes.c_double),
                ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    """gqm_tuning: launch shape of a context's flip-flop loop (0 = default)."""
    _fields_ = [("step_grid", ctypes.c_int), ("small_limit", ctypes.c_int), ("small_cluster", ctypes.c_int),
                ("check_blocks_per_sm", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


ARITH_SEPARATE, ARITH_CONTRACTED = 0, 1


def arithmetic() -> int:
    """ARITH_SEPARATE or ARITH_CONTRACTED: how the loaded library's refiner
    kernels round (see gqm_arithmetic in include/gqm_refine.h)."""
    return int(lib().gqm_arithmetic())


def set_default_tuning(device=0, step_grid=0, small_limit=0, small_cluster=0, check_blocks_per_sm=0):
    """Launch shape of the context refine() uses on `device` (gqm_set_default_tuning)."""
    t = Tuning(step_grid, small_limit, small_cluster, check_blocks_per_sm)
    rc = lib().gqm_set_default_tuning(int(device), ctypes.byref(t))
    if rc != 0:
        raise RefineError(rc, lib().gqm_status_string(rc).decode())


def use_library(path):
    """Load the refiner from another in-tree build (e.g. libgqm_b200_fma.so,
    the contracted-arithmetic variant) for the calls that follow."""
    global _lib
    _native.CUDA_LIB = path
    _lib = None
    return lib()


class RefineError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """The sm_100a library; raises when it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_native.CUDA_LIB):
            raise RuntimeError(f"{_native.CUDA_LIB} is missing: run `python -m gpu_cdt_refine_b200.build`")
        L = ctypes.CDLL(_native.CUDA_LIB)
        L.gqm_default_options.argtypes = [ctypes.POINTER(Options)]
        L.gqm_refine.argtypes = [ctypes.POINTER(CdtIn), ctypes.POINTER(CdtOut), ctypes.POINTER(Options),
                                 ctypes.POINTER(Stats)]
        L.gqm_refine.restype = ctypes.c_int
        L.gqm_free_result.argtypes = [ctypes.POINTER(CdtOut)]
        L.gqm_status_string.argtypes = [ctypes.c_int]
        L.gqm_status_string.restype = ctypes.c_char_p
        L.gqm_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.gqm_context_create.restype = ctypes.c_int
        L.gqm_context_destroy.argtypes = [ctypes.c_void_p]
        L.gqm_context_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(CdtIn), ctypes.c_int,
                                      ctypes.POINTER(Options), ctypes.POINTER(Stats)]
        L.gqm_context_run.restype = ctypes.c_int
        L.gqm_context_result.argtypes = [ctypes.c_void_p, ctypes.POINTER(CdtOut)]
        L.gqm_context_result.restype = ctypes.c_int
        L.gqm_context_result_sizes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.gqm_context_result_sizes.restype = ctypes.c_int
        L.gqm_context_stream.argtypes = [ctypes.c_void_p]
        L.gqm_context_stream.restype = ctypes.c_void_p
        L.gqm_version.restype = ctypes.c_int
        L.gqm_refine_batch.argtypes = [ctypes.c_int, ctypes.POINTER(CdtIn), ctypes.POINTER(CdtOut),
                                       ctypes.POINTER(Options), ctypes.POINTER(Stats), ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int)]
        L.gqm_refine_batch.restype = ctypes.c_int
        L.gqm_context_flip_profile.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong)]
        L.gqm_context_flip_profile.restype = ctypes.c_int
        L.gqm_refine_batch_persistent.argtypes = [ctypes.c_int, ctypes.POINTER(CdtIn), ctypes.POINTER(CdtOut),
                                                  ctypes.POINTER(Options), ctypes.POINTER(Stats),
                                                  ctypes.POINTER(BatchOptions), ctypes.POINTER(BatchReport),
                                                  ctypes.POINTER(ctypes.c_int)]
        L.gqm_refine_batch_persistent.restype = ctypes.c_int
        L.gqm_batch_autotune.argtypes = [ctypes.c_int, ctypes.POINTER(CdtIn), ctypes.POINTER(Options),
                                         ctypes.POINTER(BatchOptions), ctypes.POINTER(ctypes.c_double)]
        L.gqm_batch_autotune.restype = ctypes.c_int
        L.gqm_batch_variants.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.gqm_batch_variants.restype = ctypes.c_int
        L.gqm_batch_release.argtypes = [ctypes.c_int]
        fp = ctypes.POINTER(ctypes.c_float)
        L.gqm_learn_collect.argtypes = [ctypes.POINTER(CdtIn), ctypes.POINTER(Options), fp, fp, ctypes.c_longlong,
                                        ctypes.POINTER(ctypes.c_longlong)]
        L.gqm_learn_collect.restype = ctypes.c_int
        ip = ctypes.POINTER(ctypes.c_int)
        L.gqm_learn_explore.argtypes = [ctypes.POINTER(CdtIn), ctypes.POINTER(Options), ctypes.c_int, ctypes.c_uint,
                                        fp, ctypes.c_float, fp, ip, fp, ip, ctypes.POINTER(ctypes.c_ubyte), ip,
                                        ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
        L.gqm_learn_explore.restype = ctypes.c_int
        if hasattr(L, "gqm_mlp_infer"):  # absent from the CPU emulation build of the tests
            L.gqm_mlp_infer.argtypes = [ctypes.c_int, fp, fp, ctypes.c_longlong, fp]
            L.gqm_mlp_infer.restype = ctypes.c_int
            L.gqm_mlp_grad.argtypes = [ctypes.c_int, fp, fp, fp, ctypes.c_longlong, fp, fp]
            L.gqm_mlp_grad.restype = ctypes.c_int
            L.gqm_mlp_train.argtypes = [ctypes.c_int, fp, fp, fp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_float, ctypes.c_uint, fp]
            L.gqm_mlp_train.restype = ctypes.c_int
            L.gqm_mlp_time.argtypes = [ctypes.c_int, fp, ctypes.c_longlong, ctypes.c_int, fp]
            L.gqm_mlp_time.restype = ctypes.c_int
        L.gqm_context_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
        L.gqm_context_set_tuning.restype = ctypes.c_int
        L.gqm_context_get_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
        L.gqm_context_get_tuning.restype = ctypes.c_int
        L.gqm_context_autotune.argtypes = [ctypes.c_void_p, ctypes.POINTER(CdtIn), ctypes.c_int,
                                           ctypes.POINTER(Options), ctypes.c_int, ctypes.POINTER(Tuning),
                                           ctypes.POINTER(ctypes.c_double)]
        L.gqm_context_autotune.restype = ctypes.c_int
        L.gqm_arithmetic.restype = ctypes.c_int
        L.gqm_set_default_tuning.argtypes = [ctypes.c_int, ctypes.POINTER(Tuning)]
        L.gqm_set_default_tuning.restype = ctypes.c_int
        L.gqm_context_probe.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.gqm_context_probe.restype = ctypes.c_int
        L.gqm_context_probe_read.argtypes = [ctypes.c_void_p, ctypes.POINTER(Probe)]
        L.gqm_context_probe_read.restype = ctypes.c_int
        _lib = L
    return _lib


PLACE_PLAIN, PLACE_LEARNED = 0, 1
MLP_FEATURES, MLP_PARAMS = 32, 6337


def make_options(theta=20.0, insertpolicy=Offcenter, mode=1, predicates=PRED_REFERENCE, device=0,
                 max_rounds=0, mlp=None, max_area=0.0) -> Options:
    """Options of one refinement.  mlp: a float32 array of MLP_PARAMS network
    parameters selects the learned Steiner placement (the caller keeps the
    array alive while the options are in use)."""
    o = Options()
    lib().gqm_default_options(ctypes.byref(o))
    o.theta = float(theta)
    o.insert_policy = int(insertpolicy)
    o.mode = 1 if mode else 0
    o.predicates = int(predicates)
    o.device = int(device)
    o.max_rounds = int(max_rounds)
    o.max_area = float(max_area)
    if mlp is not None:
        if mlp.dtype != np.float32 or mlp.shape != (MLP_PARAMS,) or not mlp.flags.c_contiguous:
            raise ValueError("mlp must be a contiguous float32 array of MLP_PARAMS values")
        o.placement = PLACE_LEARNED
        o.mlp = mlp.ctypes.data
    return o


def _cdt_in(cdt: CDT, keep):
    arrs = [np.ascontiguousarray(cdt.pointlist, np.float64), np.ascontiguousarray(cdt.trianglelist, np.int32),
            np.ascontiguousarray(cdt.neighborlist, np.int32), np.ascontiguousarray(cdt.segmentlist, np.int32)]
    keep.extend(arrs)
    return CdtIn(arrs[0].shape[0], arrs[0].ctypes.data, arrs[1].shape[0], arrs[1].ctypes.data, arrs[2].ctypes.data,
                 arrs[3].shape[0], arrs[3].ctypes.data)


class _Owner:
    """Owns one gqm_cdt_out; releases it (gqm_free_result) when the last numpy
    array viewing its memory is gone."""

    def __init__(self, L, out: CdtOut):
        self._L, self._out = L, out

    def __del__(self):
        try:
            self._L.gqm_free_result(ctypes.byref(self._out))
        except Exception:
            pass


class _Mem:
    """numpy's handle on library memory at addr: the array's base, so the
    library's memory (its owner) lives as long as the array."""

    __slots__ = ("__array_interface__", "_owner")

    def __init__(self, addr, shape, typestr, owner):
        self.__array_interface__ = {"data": (addr, False), "shape": shape, "typestr": typestr, "version": 3}
        self._owner = owner


_F64, _I32, _U8 = np.dtype(np.float64).str, np.dtype(np.int32).str, np.dtype(np.uint8).str
_EMPTY = {_F64: np.float64, _I32: np.int32, _U8: np.uint8}


def _view(owner, addr, shape, typestr):
    # an array interface over the address, not a ctypes array type per length
    # (several times faster for the thousands of small arrays of a batch)
    if not addr or shape[0] == 0:
        return np.zeros(shape, _EMPTY[typestr])
    return np.asarray(_Mem(addr, shape, typestr, owner))


def _take(out: CdtOut, with_status=False, L=None):
    """numpy arrays of a result.  With L (the library), the arrays view the
    library's own memory and take over its release (no copy): the caller must
    then not call gqm_free_result on `out`.  Without L they are copies."""
    np_, nt_, ns_ = out.numberofpoints, out.numberoftriangles, out.numberofsegments
    if L is not None:
        own = _Owner(L, out)
        a = _CdtOutAddr.from_buffer(out)
        res = CDT.wrap(_view(own, a.pointlist, (np_, 2), _F64), _view(own, a.trianglelist, (nt_, 3), _I32),
                       _view(own, a.neighborlist, (nt_, 3), _I32), _view(own, a.segmentlist, (ns_, 2), _I32))
        if not with_status:
            return res
        return res, _view(own, a.pstatus, (np_,), _U8), _view(own, a.tstatus, (nt_,), _U8)
    res = CDT(np.ctypeslib.as_array(out.pointlist, shape=(2 * np_,)).copy() if np_ else np.zeros(0),
              np.ctypeslib.as_array(out.trianglelist, shape=(3 * nt_,)).copy() if nt_ else np.zeros(0, np.int32),
              np.ctypeslib.as_array(out.neighborlist, shape=(3 * nt_,)).copy() if nt_ else np.zeros(0, np.int32),
              np.ctypeslib.as_array(out.segmentlist, shape=(2 * ns_,)).copy() if ns_ else np.zeros(0, np.int32))
    if not with_status:
        return res
    ps = np.ctypeslib.as_array(out.pstatus, shape=(np_,)).copy() if np_ else np.zeros(0, np.uint8)
    ts = np.ctypeslib.as_array(out.tstatus, shape=(nt_,)).copy() if nt_ else np.zeros(0, np.uint8)
    return res, ps, ts


def refine(cdt: CDT, theta=20.0, insertpolicy=Offcenter, mode=1, predicates=PRED_REFERENCE, device=0,
           max_rounds=0, with_status=False, mlp=None, max_area=0.0):
    """Refine a CDT on the GPU; returns (CDT, stats dict) or (CDT, ps, ts, stats).
    max_area > 0 also refines every triangle larger than max_area."""
    L = lib()
    keep = []
    cin = _cdt_in(cdt, keep)
    out = CdtOut()
    st = Stats()
    opt = make_options(theta, insertpolicy, mode, predicates, device, max_rounds, mlp, max_area)
    rc = L.gqm_refine(ctypes.byref(cin), ctypes.byref(out), ctypes.byref(opt), ctypes.byref(st))
    if rc != 0:
        raise RefineError(rc, L.gqm_status_string(rc).decode())
    got = _take(out, with_status, L)  # the arrays own the library's memory from here
    if with_status:
        return (*got, st.as_dict())
    return got, st.as_dict()


def refine_batch(cdts, thetas=20.0, insertpolicy=Offcenter, mode=1, predicates=PRED_REFERENCE, device=0,
                 workers=8, max_rounds=0):
    """Refine independent CDTs concurrently (gqm_refine_batch); returns
    (list of CDT, list of stats dicts)."""
    L = lib()
    n = len(cdts)
    if np.isscalar(thetas):
        thetas = [float(thetas)] * n
    keep = []
    ins = (CdtIn * n)(*[_cdt_in(c, keep) for c in cdts])
    outs = (CdtOut * n)()
    opts = (Options * n)(*[make_options(t, insertpolicy, mode, predicates, device, max_rounds) for t in thetas])
    sts = (Stats * n)()
    bad = ctypes.c_int(-1)
    rc = L.gqm_refine_batch(n, ins, outs, opts, sts, int(workers), ctypes.byref(bad))
    if rc != 0:
        for i in range(n):
            L.gqm_free_result(ctypes.byref(outs[i]))
        raise RefineError(rc, f"domain {bad.value}: " + L.gqm_status_string(rc).decode())
    res = [_take(outs[i], L=L) for i in range(n)]  # each result owns its domain's memory
    return res, [sts[i].as_dict() for i in range(n)]


def _batch_args(cdts, thetas, insertpolicy, mode, predicates, device, max_rounds, keep, mlp=None, max_area=0.0):
    n = len(cdts)
    if np.isscalar(thetas):
        thetas = [float(thetas)] * n
    if np.isscalar(predicates):
        predicates = [int(predicates)] * n
    ins = (CdtIn * n)(*[_cdt_in(c, keep) for c in cdts])
    made = {}  # one Options per distinct (theta, predicates), copied into the array
    for t, p in zip(thetas, predicates):
        if (t, p) not in made:
            made[(t, p)] = make_options(t, insertpolicy, mode, p, device, max_rounds, mlp, max_area)
    opts = (Options * n)(*[made[(t, p)] for t, p in zip(thetas, predicates)])
    return ins, opts


def refine_batch_persistent(cdts, thetas=20.0, insertpolicy=Offcenter, mode=1, predicates=PRED_REFERENCE, device=0,
                            threads_per_block=0, blocks_per_sm=0, max_rounds=0, with_report=False, mlp=None,
                            max_area=0.0):
    """Refine independent CDTs in one persistent launch
    (gqm_refine_batch_persistent); returns (list of CDT, list of stats dicts)
    and, with with_report, the call's report as a third item."""
    L = lib()
    n = len(cdts)
    keep = []
    ins, opts = _batch_args(cdts, thetas, insertpolicy, mode, predicates, device, max_rounds, keep, mlp, max_area)
    outs = (CdtOut * n)()
    sts = (Stats * n)()
    bo = BatchOptions(int(threads_per_block), int(blocks_per_sm), 0.0)
    rep = BatchReport()
    bad = ctypes.c_int(-1)
    rc = L.gqm_refine_batch_persistent(n, ins, outs, opts, sts, ctypes.byref(bo), ctypes.byref(rep),
                                       ctypes.byref(bad))
    if rc != 0:
        for i in range(n):
            L.gqm_free_result(ctypes.byref(outs[i]))
        raise RefineError(rc, f"domain {bad.value}: " + L.gqm_status_string(rc).decode())
    res = [_take(outs[i], L=L) for i in range(n)]  # each result owns its domain's memory
    stats = [sts[i].as_dict() for i in range(n)]
    if with_report:
        return res, stats, rep.as_dict()
    return res, stats


def batch_variants():
    """The compiled (threads per block, blocks per SM) pairs of the batch kernel."""
    L = lib()
    t, b = (ctypes.c_int * 16)(), (ctypes.c_int * 16)()
    n = L.gqm_batch_variants(t, b, 16)
    return [(t[i], b[i]) for i in range(n)]


def batch_autotune(cdts, thetas=20.0, insertpolicy=Offcenter, mode=1, predicates=PRED_REFERENCE, device=0):
    """Time every batch kernel variant on `cdts` and keep the fastest for later
    calls on `device`; returns ((threads, blocks per SM), {variant: kernel ms})."""
    L = lib()
    keep = []
    ins, opts = _batch_args(cdts, thetas, insertpolicy, mode, predicates, device, 0, keep)
    chosen = BatchOptions()
    ms = (ctypes.c_double * 16)()
    rc = L.gqm_batch_autotune(len(cdts), ins, opts, ctypes.byref(chosen), ms)
    if rc != 0:
        raise RefineError(rc, "autotune: " + L.gqm_status_string(rc).decode())
    return (chosen.threads_per_block, chosen.blocks_per_sm), {v: ms[i] for i, v in enumerate(batch_variants())}


# --- learned Steiner placement ----------------------------------------------

def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_init(seed=0, t0=0.5):
    """Initial network parameters (He-scaled normal weights, zero biases, output
    bias t0) as a float32 array of MLP_PARAMS values."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_PARAMS, np.float32)
    o = 0
    p[o:o + 64 * 32] = rng.normal(0, np.sqrt(2.0 / 32), 64 * 32)
    o += 64 * 32 + 64
    p[o:o + 64 * 64] = rng.normal(0, np.sqrt(2.0 / 64), 64 * 64)
    o += 64 * 64 + 64
    p[o:o + 64] = rng.normal(0, np.sqrt(1.0 / 64), 64) * 0.1
    p[-1] = t0
    return p


def learn_collect(cdt: CDT, theta=20.0, insertpolicy=Offcenter, mode=1, device=0, cap=1_000_000):
    """Training rows from a plain refinement of `cdt` (gqm_learn_collect):
    (features [n, 32] float32, targets [n] float32)."""
    L = lib()
    keep = []
    cin = _cdt_in(cdt, keep)
    opt = make_options(theta, insertpolicy, mode, PRED_REFERENCE, device)
    feat = np.zeros((cap, MLP_FEATURES), np.float32)
    tgt = np.zeros(cap, np.float32)
    cnt = ctypes.c_longlong(0)
    rc = L.gqm_learn_collect(ctypes.byref(cin), ctypes.byref(opt), _fp(feat), _fp(tgt), int(cap), ctypes.byref(cnt))
    if rc != 0:
        raise RefineError(rc, "learn_collect: " + L.gqm_status_string(rc).decode())
    return feat[:cnt.value].copy(), tgt[:cnt.value].copy()


def learn_explore(cdt: CDT, theta=20.0, levels=5, seed=0, insertpolicy=Offcenter, mode=1, device=0, cap=None,
                  mlp=None, eps=1.0):
    """Rows of an exploration run (gqm_learn_explore): a dict of per-row arrays
    features [n, 32], level, t_used, parent, inserted, midpoints.  With a
    network, a triangle draws a level with probability eps and otherwise takes
    the network's t (level -2)."""
    L = lib()
    net = None
    if mlp is not None:
        net = np.ascontiguousarray(mlp, np.float32)
        if net.shape != (MLP_PARAMS,):
            raise ValueError("mlp must hold MLP_PARAMS values")
    keep = []
    cin = _cdt_in(cdt, keep)
    opt = make_options(theta, insertpolicy, mode, PRED_REFERENCE, device)
    cap = int(cap if cap is not None else max(1024, 4 * cdt.numberofpoints))
    for _ in range(2):
        feat = np.zeros((cap, MLP_FEATURES), np.float32)
        level = np.zeros(cap, np.int32)
        tused = np.zeros(cap, np.float32)
        parent = np.zeros(cap, np.int32)
        ins = np.zeros(cap, np.uint8)
        mids = np.zeros(cap, np.int32)
        cnt = ctypes.c_longlong(0)
        ip = ctypes.POINTER(ctypes.c_int)
        rc = L.gqm_learn_explore(ctypes.byref(cin), ctypes.byref(opt), int(levels), int(seed) & 0xFFFFFFFF,
                                 _fp(net) if net is not None else None, float(eps), _fp(feat), level.ctypes.data_as(ip), _fp(tused), parent.ctypes.data_as(ip),
                                 ins.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), mids.ctypes.data_as(ip), cap,
                                 ctypes.byref(cnt))
        if rc == -13 and cnt.value > cap:  # GQM_ERR_TOO_LARGE: run again with room for every row
            cap = int(cnt.value * 1.25) + 1024
            continue
        if rc != 0:
            raise RefineError(rc, "learn_explore: " + L.gqm_status_string(rc).decode())
        n = cnt.value
        return {"features": feat[:n].copy(), "level": level[:n].copy(), "t_used": tused[:n].copy(),
                "parent": parent[:n].copy(), "inserted": ins[:n].copy(), "midpoints": mids[:n].copy()}
    raise RefineError(-13, "learn_explore: rows outgrew the capacity twice")


def descendants(parent, inserted, midpoints, depth=0):
    """Descendant count of every row of an exploration run: the inserted rows
    and the midpoints below it in the parent tree, down to `depth` generations
    (0: all).  Parents precede their children (a parent row is a vertex of an
    earlier round), so one pass from the last row back sums whole subtrees."""
    parent = np.asarray(parent, np.int64)
    own = np.asarray(midpoints, np.float64)
    ins = np.asarray(inserted, np.float64)
    n = parent.shape[0]
    if n and parent.max(initial=-1) >= n:
        raise ValueError("parent row out of range")
    has = parent >= 0
    if np.any(parent[has] >= np.arange(n)[has]):
        raise ValueError("a parent row must precede its child")
    if depth <= 0:
        d = own.copy()
        for r in range(n - 1, -1, -1):  # children before parents
            p = parent[r]
            if p >= 0:
                d[p] += ins[r] + d[r]
        return d
    # a[r]: descendants exactly k generations below r (the row's own midpoints
    # and inserted children are generation 1)
    a = own + np.bincount(parent[has], weights=ins[has], minlength=n)
    total = a.copy()
    for _ in range(depth - 1):
        a = np.bincount(parent[has], weights=a[has], minlength=n)
        total += a
    return total


def mlp_infer(params, features, device=0):
    L = lib()
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32)
    out = np.zeros(x.shape[0], np.float32)
    rc = L.gqm_mlp_infer(int(device), _fp(p), _fp(x), x.shape[0], _fp(out))
    if rc != 0:
        raise RefineError(rc, "mlp_infer")
    return out


def mlp_grad(params, features, targets, device=0):
    """(loss, gradient) of the mean squared error on the GPU."""
    L = lib()
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    rc = L.gqm_mlp_grad(int(device), _fp(p), _fp(x), _fp(t), x.shape[0], _fp(loss), _fp(g))
    if rc != 0:
        raise RefineError(rc, "mlp_grad")
    return float(loss[0]), g


def mlp_train(params, features, targets, epochs=20, batch=256, lr=1e-3, seed=0, device=0):
    """Adam training on the GPU; returns (trained params, last epoch's loss)."""
    L = lib()
    p = np.array(params, np.float32, copy=True)
    x = np.ascontiguousarray(features, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    loss = np.zeros(1, np.float32)
    rc = L.gqm_mlp_train(int(device), _fp(p), _fp(x), _fp(t), x.shape[0], int(epochs), int(batch), float(lr),
                         int(seed), _fp(loss))
    if rc != 0:
        raise RefineError(rc, "mlp_train")
    return p, float(loss[0])


def mlp_time(params, n, iters=10, device=0):
    """Device milliseconds of one network inference launch over n rows."""
    L = lib()
    p = np.ascontiguousarray(params, np.float32)
    ms = np.zeros(1, np.float32)
    rc = L.gqm_mlp_time(int(device), _fp(p), int(n), int(iters), _fp(ms))
    if rc != 0:
        raise RefineError(rc, "mlp_time")
    return float(ms[0])


def GPU_Refine_Quality(input: CDT, theta: float, insertpolicy=Offcenter, deletepolicy=Connected, mode=1,
                       debug_iter=-1, ps_debug=False, ts_debug=False):
    """Drop-in for the reference entry point (GPU_Refine/refine.h:385-386).

    `deletepolicy` and `debug_iter` are accepted and ignored, as in the
    reference.  Returns the refined CDT, or (CDT, pstatus, tstatus) when
    `ps_debug` or `ts_debug` is true.
    """
    del deletepolicy, debug_iter
    want = bool(ps_debug or ts_debug)
    r = refine(input, theta, insertpolicy, mode, with_status=want)
    if want:
        return r[0], r[1], r[2]
    return r[0]


class Context:
    """Reusable device context (gqm_context): buffers persist between runs."""

    def __init__(self, device=0):
        self._lib = lib()
        self._h = ctypes.c_void_p()
        rc = self._lib.gqm_context_create(int(device), ctypes.byref(self._h))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())

    def close(self):
        if self._h:
            self._lib.gqm_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self._lib.gqm_context_stream(self._h) or 0)

    def run_device(self, np_, nt_, ns_, d_points, d_tris, d_nbrs, d_segs, opt: Options) -> dict:
        """Refine inputs that already live in device memory (raw pointers)."""
        cin = CdtIn(np_, d_points, nt_, d_tris, d_nbrs, ns_, d_segs)
        st = Stats()
        rc = self._lib.gqm_context_run(self._h, ctypes.byref(cin), 1, ctypes.byref(opt), ctypes.byref(st))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())
        return st.as_dict()

    def run_host(self, cdt: CDT, opt: Options) -> dict:
        keep = []
        cin = _cdt_in(cdt, keep)
        st = Stats()
        rc = self._lib.gqm_context_run(self._h, ctypes.byref(cin), 0, ctypes.byref(opt), ctypes.byref(st))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())
        return st.as_dict()

    def sizes(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = self._lib.gqm_context_result_sizes(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        if rc != 0:
            raise RefineError(rc, "no result")
        return a.value, b.value, c.value

    def flip_profile(self):
        """(steps, items) per floor(log2 |active set|) bin of the last run's flip steps."""
        st, it = (ctypes.c_longlong * 32)(), (ctypes.c_longlong * 32)()
        rc = self._lib.gqm_context_flip_profile(self._h, st, it)
        if rc != 0:
            raise RefineError(rc, "flip profile")
        return list(st), list(it)

    def set_tuning(self, step_grid=0, small_limit=0, small_cluster=0, check_blocks_per_sm=0):
        """Launch shape of the flip-flop loop (gqm_context_set_tuning); 0 keeps
        a field's default, small_limit < 0 turns the small-step kernel off."""
        t = Tuning(step_grid, small_limit, small_cluster, check_blocks_per_sm)
        rc = self._lib.gqm_context_set_tuning(self._h, ctypes.byref(t))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())

    def tuning(self) -> dict:
        t = Tuning()
        rc = self._lib.gqm_context_get_tuning(self._h, ctypes.byref(t))
        if rc != 0:
            raise RefineError(rc, "tuning")
        return t.as_dict()

    def autotune(self, cdt: CDT, opt: Options, repeats=1):
        """gqm_context_autotune on a host-array input: returns (chosen shape, its ms)."""
        keep = []
        cin = _cdt_in(cdt, keep)
        t, ms = Tuning(), ctypes.c_double()
        rc = self._lib.gqm_context_autotune(self._h, ctypes.byref(cin), 0, ctypes.byref(opt), int(repeats),
                                            ctypes.byref(t), ctypes.byref(ms))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())
        return t.as_dict(), ms.value

    def probe(self, enable=True):
        """Reset and enable (or disable) the launch timer of the flip-step check
        kernel and the events around the flip-loop launches."""
        rc = self._lib.gqm_context_probe(self._h, 1 if enable else 0)
        if rc != 0:
            raise RefineError(rc, "probe")

    def probe_read(self) -> dict:
        p = Probe()
        rc = self._lib.gqm_context_probe_read(self._h, ctypes.byref(p))
        if rc != 0:
            raise RefineError(rc, "probe read")
        return p.as_dict()

    def result(self, with_status=False):
        out = CdtOut()
        rc = self._lib.gqm_context_result(self._h, ctypes.byref(out))
        if rc != 0:
            raise RefineError(rc, self._lib.gqm_status_string(rc).decode())
        try:
            return _take(out, with_status)
        finally:
            self._lib.gqm_free_result(ctypes.byref(out))
