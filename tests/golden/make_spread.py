"""Generate the run-to-run spread of the reference GPU refiner (test fixture).

Needs a CUDA GPU and the reference build (`make -C oracle ref`):

    python tests/golden/make_spread.py [OUT_JSON]

For every configuration of tests/golden/reference_outputs.json (same seeded
inputs, same theta / policy / mode), the reference's own GPU_Refine_Quality
(GPU_Refine/refine.h:385-386), compiled from its sources by oracle/Makefile, is
run again many times, each run a process of its own:

* gqm_ref_run_nofma (-fmad=false), NOFMA_RUNS times for the configurations
  whose runs differ: the output sizes of every run (the reference's output
  varies with which of two racing subseg2tri stores lands,
  GPU_Refine/refine.cu:1362-1372 and the like);
* gqm_ref_run (the reference as its project builds it: nvcc's default FMA
  contraction), FMA_RUNS times for every configuration: the sizes and digests
  of every run, and whether all runs agree byte for byte.

Runs go WORKERS at a time on the one GPU (independent processes; nothing
waits on another).
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import ROOT, make_input, run_ref, summary  # noqa: E402

from gpu_cdt_refine_b200 import cdtio  # noqa: E402

NOFMA_RUNS = 12
FMA_RUNS = 6
WORKERS = 4


def main():
    out_json = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_spread.json")
    with open(os.path.join(HERE, "reference_outputs.json")) as f:
        gold = json.load(f)
    doc = {"note": "run-to-run spread of the reference GPU_Refine_Quality built from its own sources; "
                   "see make_spread.py", "nofma_runs": NOFMA_RUNS, "fma_runs": FMA_RUNS, "cases": {}}
    with tempfile.TemporaryDirectory() as d, cf.ThreadPoolExecutor(WORKERS) as pool:
        jobs = []
        for name, case in gold["cases"].items():
            path = os.path.join(d, name + ".bin")
            cdtio.write_cdt(path, make_input(name))
            for k, cfg in enumerate(case["configs"]):
                key = (name, k)
                args = (path, cfg["theta"], cfg["policy"], cfg["mode"])
                if not cfg["self_consistent"]:
                    jobs += [(key, "nofma", pool.submit(run_ref, "gqm_ref_run_nofma", *args)) for _ in range(NOFMA_RUNS)]
                jobs += [(key, "fma", pool.submit(run_ref, "gqm_ref_run", *args)) for _ in range(FMA_RUNS)]
        res = {}
        for key, kind, fut in jobs:
            out, _ = fut.result()
            res.setdefault(key, {"nofma": [], "fma": []})[kind].append(summary(out))
    for name, case in gold["cases"].items():
        cfgs = []
        for k, cfg in enumerate(case["configs"]):
            r = res[(name, k)]
            fma = r["fma"]
            entry = {"theta": cfg["theta"], "policy": cfg["policy"], "mode": cfg["mode"],
                     "nofma_sizes": [[x["points"], x["triangles"], x["segments"]] for x in r["nofma"]],
                     "fma_sizes": [[x["points"], x["triangles"], x["segments"]] for x in fma],
                     "fma_self_consistent": all(x["sha256"] == fma[0]["sha256"] for x in fma),
                     "fma_sha256": fma[0]["sha256"]}
            cfgs.append(entry)
            print(name, cfg["theta"], cfg["policy"], cfg["mode"], "fma consistent" if entry["fma_self_consistent"]
                  else "fma varies", sorted({tuple(s) for s in entry["nofma_sizes"]}), flush=True)
        doc["cases"][name] = cfgs
    with open(out_json, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", out_json)


if __name__ == "__main__":
    main()
