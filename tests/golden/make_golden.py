"""Generate the golden outputs of the reference GPU refiner (test fixtures).

Needs a CUDA GPU and the reference build (`make -C oracle ref`):

    python tests/golden/make_golden.py [OUT_JSON]

Every input CDT below comes from the package's seeded generators and is
refined by the reference's own GPU_Refine_Quality (GPU_Refine/refine.h:385-386)
through oracle/_ref/gqm_ref_run_nofma (GPU_Refine/refine.cu compiled unmodified
with -fmad=false) and oracle/_ref/gqm_ref_run (nvcc's default FMA contraction).
Each output array is recorded as a SHA-256 digest of its raw little-endian
bytes, with the output sizes and the reference's wall time.

cos^2(theta) is recorded as CUDA's device cos() evaluates it (the reference
computes it inside its kernels, GPU_Refine/refine.cu:418-419), so that the CPU
oracle can be given the same value.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpu_cdt_refine_b200 import cdtio, inputs  # noqa: E402

FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")
CFG4 = [(20.0, 1, 1), (20.0, 1, 0), (20.0, 0, 1), (20.0, 0, 0)]

# name -> (generator expression, [(theta, policy, mode)], size class)
# "small" cases are checked against the CPU oracle as well as the GPU path.
# Inputs stay below the 1,280,000 input triangles up to which the reference's
# initSubsegs is correct (GPU_Refine/refine.cu:5691-5747), and away from
# near-degenerate point sets: the reference's point-location walk has no
# iteration bound (refine.cu:4036) and its predicates are inexact, so a
# near-degenerate input could keep one of its kernels running indefinitely.
CASES = {
    "u2k": ("inputs.plain_small(seed=201, n=2000, nseg=100)", CFG4 + [(15.0, 1, 1), (25.0, 1, 1)], "small"),
    "u5k": ("inputs.plain_small(seed=202, n=5000, nseg=600)", CFG4, "small"),
    "cl8k": ("inputs.clustered(seed=203, n=8000, nseg=400)", CFG4, "small"),
    "c1": ("inputs.plain_small()", CFG4, "small"),
    "u100k": ("inputs.plain_small(seed=211, n=100000, nseg=5000)", CFG4, "medium"),
    "cl500k": ("inputs.clustered(seed=31, n=500000, nseg=25000)", [(20.0, 1, 1)], "medium"),
}


def make_input(name):
    return eval(CASES[name][0], {"inputs": inputs})


def digests(cdt):
    return {f: hashlib.sha256(np.ascontiguousarray(getattr(cdt, f)).tobytes()).hexdigest() for f in FIELDS}


def device_goodcos2(theta):
    """cos^2(theta) from the refiner's one-thread device evaluation."""
    from gpu_cdt_refine_b200 import refine
    c = inputs.plain_small(seed=1, n=50, nseg=2)
    _, st = refine.refine(c, theta, refine.Offcenter, 1)
    return st["goodcos2"]


def run_ref(binary, path_in, theta, policy, mode, reps=3):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        p = subprocess.run([os.path.join(ROOT, "oracle", "_ref", binary), path_in, out, repr(theta), str(policy),
                            str(mode), str(reps)], capture_output=True, text=True, timeout=600)
        if p.returncode != 0:
            raise RuntimeError(f"{binary} failed ({p.returncode}): {p.stderr[-500:]}")
        info = json.loads([l for l in p.stderr.splitlines() if l.startswith("GQMREF ")][0][7:])
        res = cdtio.read_cdt(out)
    return res, info


def main():
    out_json = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "reference_outputs.json")
    doc = {"note": "outputs of the reference GPU_Refine_Quality built from its own sources; see make_golden.py",
           "device_goodcos2": {}, "cases": {}}
    thetas = sorted({t for _, cfgs, _ in CASES.values() for t, _, _ in cfgs})
    for t in thetas:
        doc["device_goodcos2"][repr(t)] = device_goodcos2(t)
    with tempfile.TemporaryDirectory() as d:
        for name, (expr, cfgs, size) in CASES.items():
            cdt = make_input(name)
            path = os.path.join(d, name + ".bin")
            cdtio.write_cdt(path, cdt)
            case = {"generator": expr, "size": size,
                    "input": {"points": cdt.numberofpoints, "triangles": cdt.numberoftriangles,
                              "segments": cdt.numberofsegments, "sha256": digests(cdt)}, "runs": []}
            for theta, policy, mode in cfgs:
                for binary, arith in (("gqm_ref_run_nofma", "nofma"), ("gqm_ref_run", "fma")):
                    res, info = run_ref(binary, path, theta, policy, mode)
                    case["runs"].append({"theta": theta, "policy": policy, "mode": mode, "arith": arith,
                                         "points": res.numberofpoints, "triangles": res.numberoftriangles,
                                         "segments": res.numberofsegments, "sha256": digests(res),
                                         "ms": info["ms"]})
                    print(name, theta, policy, mode, arith, res.numberoftriangles, info["ms"], flush=True)
            doc["cases"][name] = case
    with open(out_json, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", out_json)


if __name__ == "__main__":
    main()
