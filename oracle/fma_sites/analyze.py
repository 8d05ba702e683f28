"""Which products the reference's own build fuses (test infrastructure).

    make -C oracle fma-probes                      # here: builds the probes and candidates
    oracle/_ref/fma_probe_predicates P.bin         # on a B200
    oracle/_ref/fma_probe_kernels K.bin            # on a B200
    python oracle/fma_sites/analyze.py P.bin K.bin

For every expression of the reference's arithmetic that contains a product
consumed by an add or subtract, each candidate evaluation (candidates.c:
unfused, first product fused, second product fused; per term where the terms
can differ) is compared bit for bit with the outputs of the reference's
compiled predicates and kernels; the candidate that reproduces every output
is the reference build's arithmetic.  The contracted oracle (madd() in
oracle/gqm_oracle.c) and the contracted library (gqm_madd() in
gpu_cdt_refine_b200/csrc) use exactly these.
"""
from __future__ import annotations

import collections
import ctypes
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "_build", "libfma_candidates.so")
DP = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return np.ascontiguousarray(a).ctypes.data_as(DP)


def predicates(path, C, m=20000):
    n = 200000
    raw = open(path, "rb").read()
    pts = np.frombuffer(raw[:n * 64], dtype=np.float64).reshape(n, 4, 2)
    out = np.frombuffer(raw[n * 64:], dtype=np.float64).reshape(n, 4)
    C.ccw_v.argtypes = [DP, DP, DP, ctypes.c_int]
    C.ccw_v.restype = ctypes.c_double
    C.inc_v.argtypes = [DP, DP, DP, DP, ctypes.c_int]
    C.inc_v.restype = ctypes.c_double
    for col, name in ((0, "cuda_ccw"), (1, "cuda_fast")):
        ok = collections.Counter()
        for i in range(m):
            a, b, c = (_ptr(pts[i, k]) for k in range(3))
            for v in range(3):
                ok[v] += C.ccw_v(a, b, c, v) == out[i, col]
        print(f"{name}: matches per candidate (0 unfused, 1 first fused, 2 second fused) {dict(ok)} of {m}")
    ok = collections.Counter()
    vs = [v for v in range(64) if (v & 3) < 3 and ((v >> 2) & 3) < 3 and ((v >> 4) & 7) < 6]
    for i in range(m):
        a, b, c, d = (_ptr(pts[i, k]) for k in range(4))
        for v in vs:
            ok[v] += C.inc_v(a, b, c, d, v) == out[i, 2]
    v, k = ok.most_common(1)[0]
    print(f"cuda_inCircle: best candidate cross {v & 3} lifts {(v >> 2) & 3} sum {(v >> 4) & 7}: {k} of {m}")


def kernels(path, C, m=4000):
    n = 100000
    raw = open(path, "rb").read()
    off = 0

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(raw, dtype=dt, count=cnt, offset=off)
        off += a.nbytes
        return a

    P1 = take(np.float64, 6 * n).reshape(n, 3, 2)
    CC3 = take(np.float64, 2 * n).reshape(n, 2)
    CC2 = take(np.float64, 2 * n).reshape(n, 2)
    CCc = take(np.float64, 2 * n).reshape(n, 2)
    P2 = take(np.float64, 6 * n).reshape(n, 3, 2)
    TS = take(np.uint8, n)
    P3, ENC = [], []
    for _ in range(2):
        P3.append(take(np.float64, 6 * n).reshape(n, 3, 2))
        ENC.append(take(np.int32, n))
    C.cc_cand.argtypes = [DP, DP, DP, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int), DP]
    C.enc_cand.argtypes = [DP, DP, DP, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    C.enc_cand.restype = ctypes.c_int
    out = (ctypes.c_double * 2)()
    # circumcenter: the distances, the denominator and the two numerators
    res = collections.Counter()
    for opt in itertools.product(range(3), repeat=4):
        o = (ctypes.c_int * 7)(*opt, 0, 0, 0)
        ok = 0
        for i in range(m):
            C.cc_cand(_ptr(P1[i, 0]), _ptr(P1[i, 1]), _ptr(P1[i, 2]), 2.0, 0, o, out)
            ok += out[0] == CCc[i, 0] and out[1] == CCc[i, 1]
        res[opt] = ok
    opt, k = res.most_common(1)[0]
    print(f"circumcenter: distances {opt[0]} denominator {opt[1]} numerators {opt[2:]}: {k} of {m}")
    score = (ctypes.c_int * 576)()
    C.off_search.argtypes = [DP, DP, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    for offc, cc in ((3.0, CC3), (2.0, CC2)):
        C.off_search(_ptr(P1), _ptr(cc), 20000, offc, score, None)
        best = max(range(576), key=lambda k: score[k])
        o, t = [], best
        for _ in range(6):
            o.append(t % 2)
            t //= 2
        print(f"off-center (offConstant {offc:g}): branches {o} comparisons {[t % 3, t // 3]}: "
              f"{score[best]} of 20000")
    bad = ((TS >> 1) & 1).astype(np.uint8)
    s3 = (ctypes.c_int * 729)()
    C.bad_search.argtypes = [DP, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.c_double,
                             ctypes.POINTER(ctypes.c_int)]
    C.bad_search(_ptr(P2), np.ascontiguousarray(bad).ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), n,
                 0.8830222215594891, s3)
    best = max(range(729), key=lambda k: s3[k])
    o, t = [], best
    for _ in range(6):
        o.append(t % 3)
        t //= 3
    print(f"smallest angle: lengths {o[:3]} dot products {o[3:]}: {s3[best]} of {n}")
    gcs = float(np.cos(20.0 * np.pi / 180.0) ** 2)
    for mode in range(2):
        enc = (ENC[mode] == 0).astype(int)
        res = collections.Counter()
        for opt in itertools.product(range(3), range(3)):
            o = (ctypes.c_int * 2)(*opt)
            res[opt] = sum(C.enc_cand(_ptr(P3[mode][i, 1]), _ptr(P3[mode][i, 2]), _ptr(P3[mode][i, 0]), gcs, mode, o)
                           == enc[i] for i in range(20000))
        opt, k = res.most_common(1)[0]
        print(f"encroachment ({'Ruppert' if mode else 'Chew'}): dot {opt[0]} lengths {opt[1]}: {k} of 20000")


def main():
    C = ctypes.CDLL(LIB)
    predicates(sys.argv[1], C)
    kernels(sys.argv[2], C)


if __name__ == "__main__":
    main()
