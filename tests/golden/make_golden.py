"""Generate the golden outputs of the reference GPU refiner (test fixtures).

Needs a CUDA GPU and the reference build (`make -C oracle ref`):

    python tests/golden/make_golden.py [OUT_JSON]

Every input CDT below comes from the package's seeded generators and is
refined by the reference's own GPU_Refine_Quality (GPU_Refine/refine.h:385-386)
compiled from its sources by oracle/Makefile:

* gqm_ref_trace (-fmad=false, with the flip-step trace of
  oracle/ref_shim/launch_trace.cpp) is run RUNS times per configuration.  The
  reference is not deterministic: two winners of one flip or insertion launch
  can store different orientations of one subsegment into subseg2tri
  (e.g. GPU_Refine/refine.cu:1363-1372), and which store lands depends on
  timing.  For every configuration the fixture keeps
    - the digests of each run's output arrays, and whether all runs agree;
    - the number of leading flip steps on which all runs' traces agree, the
      hashes of those trace lines, and the mesh digests of the first step at
      which they part.
* gqm_ref_run_nofma (untraced) gives the wall time, gqm_ref_run (nvcc's
  default FMA contraction) the output with fused multiply-adds.

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
RUNS = 4

# name -> (generator expression, [(theta, policy, mode)], size class)
# "small" cases are traced and checked against the CPU oracle as well as the
# GPU path; "medium" ones are too large to trace every flip step.
# Inputs stay below the 1,280,000 input triangles up to which the reference's
# initSubsegs is correct (GPU_Refine/refine.cu:5691-5747), and away from
# near-degenerate point sets: the reference's point-location walk has no
# iteration bound (refine.cu:4036) and its predicates are inexact, so a
# near-degenerate input could keep one of its kernels running indefinitely.
# The "h" cases have no interior segment (only the convex hull's, which have
# one triangle each), so no two winners ever share a subsegment.
CASES = {
    "u2k": ("inputs.plain_small(seed=201, n=2000, nseg=100)", CFG4 + [(15.0, 1, 1), (25.0, 1, 1)], "small"),
    "u5k": ("inputs.plain_small(seed=202, n=5000, nseg=600)", CFG4, "small"),
    "cl8k": ("inputs.clustered(seed=203, n=8000, nseg=400)", CFG4, "small"),
    "c1": ("inputs.plain_small()", CFG4, "small"),
    "s2k": ("inputs.plain_small(seed=224, n=2000, nseg=5)", CFG4, "small"),
    "h2k": ("inputs.plain_small(seed=221, n=2000, nseg=0)", CFG4, "small"),
    "h10k": ("inputs.plain_small(seed=222, n=10000, nseg=0)", CFG4, "small"),
    "hcl8k": ("inputs.clustered(seed=223, n=8000, nseg=0)", CFG4, "small"),
    "u100k": ("inputs.plain_small(seed=211, n=100000, nseg=5000)", CFG4, "medium"),
    "h100k": ("inputs.plain_small(seed=225, n=100000, nseg=0)", [(20.0, 1, 1)], "medium"),
    "cl500k": ("inputs.clustered(seed=31, n=500000, nseg=25000)", [(20.0, 1, 1)], "medium"),
}


def make_input(name):
    return eval(CASES[name][0], {"inputs": inputs})


def digests(cdt):
    return {f: hashlib.sha256(np.ascontiguousarray(getattr(cdt, f)).tobytes()).hexdigest() for f in FIELDS}


def line_hash(line):
    return hashlib.sha256(line.strip().encode()).hexdigest()[:16]


def mesh_of(line):
    return line.strip().rsplit("mesh=", 1)[1]


def device_goodcos2(theta):
    """cos^2(theta) from the refiner's one-thread device evaluation."""
    from gpu_cdt_refine_b200 import refine
    c = inputs.plain_small(seed=1, n=50, nseg=2)
    _, st = refine.refine(c, theta, refine.Offcenter, 1)
    return st["goodcos2"]


def run_ref(binary, path_in, theta, policy, mode, reps=1, trace=None):
    env = dict(os.environ)
    if trace:
        env["GQM_REF_TRACE"] = trace
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        p = subprocess.run([os.path.join(ROOT, "oracle", "_ref", binary), path_in, out, repr(theta), str(policy),
                            str(mode), str(reps)], capture_output=True, text=True, timeout=900, env=env)
        if p.returncode != 0:
            raise RuntimeError(f"{binary} failed ({p.returncode}): {p.stderr[-500:]}")
        info = json.loads([l for l in p.stderr.splitlines() if l.startswith("GQMREF ")][0][7:])
        res = cdtio.read_cdt(out)
    return res, info


def summary(res):
    return {"points": res.numberofpoints, "triangles": res.numberoftriangles, "segments": res.numberofsegments,
            "sha256": digests(res)}


def main():
    out_json = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "reference_outputs.json")
    doc = {"note": "outputs of the reference GPU_Refine_Quality built from its own sources; see make_golden.py",
           "runs_per_config": RUNS, "device_goodcos2": {}, "cases": {}}
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
                              "segments": cdt.numberofsegments, "sha256": digests(cdt)}, "configs": []}
            for theta, policy, mode in cfgs:
                cfg = {"theta": theta, "policy": policy, "mode": mode, "runs": []}
                traces = []
                for r in range(RUNS):
                    if size == "small":
                        tp = os.path.join(d, f"trace{r}.txt")
                        res, _ = run_ref("gqm_ref_trace", path, theta, policy, mode, trace=tp)
                        traces.append([l for l in open(tp) if l.startswith("F ")])
                    else:
                        res, _ = run_ref("gqm_ref_run_nofma", path, theta, policy, mode)
                    cfg["runs"].append(summary(res))
                cfg["self_consistent"] = all(r["sha256"] == cfg["runs"][0]["sha256"] for r in cfg["runs"])
                if traces:
                    agreed = 0
                    while all(agreed < len(t) for t in traces) and len({t[agreed] for t in traces}) == 1:
                        agreed += 1
                    cfg["trace"] = {"steps": [len(t) for t in traces], "agreed_steps": agreed,
                                    "line_hashes": [line_hash(l) for l in traces[0][:agreed]],
                                    "split_meshes": [mesh_of(t[agreed]) for t in traces if agreed < len(t)]}
                _, timing = run_ref("gqm_ref_run_nofma", path, theta, policy, mode, reps=3)
                cfg["ms"] = timing["ms"]
                fma, _ = run_ref("gqm_ref_run", path, theta, policy, mode)
                cfg["fma"] = summary(fma)
                case["configs"].append(cfg)
                print(name, theta, policy, mode, "consistent" if cfg["self_consistent"] else "varies",
                      [r["triangles"] for r in cfg["runs"]], cfg.get("trace", {}).get("agreed_steps"),
                      cfg.get("trace", {}).get("steps"), cfg["ms"], flush=True)
            doc["cases"][name] = case
    with open(out_json, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", out_json)


if __name__ == "__main__":
    main()
