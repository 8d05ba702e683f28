"""The oracle against the reference's own runs.

tests/golden/reference_outputs.json (written by tests/golden/make_golden.py on
a B200) holds, for seeded inputs, the outputs of several runs of the
reference GPU_Refine_Quality built from its sources with -fmad=false, and the
digest trace of every flip step of those runs.

The reference is not deterministic: two winners of one launch can store the
two orientations of one subsegment into subseg2tri, and which store lands
depends on timing (the runs then differ in which slots the same triangles
occupy, and later in the mesh).  The oracle fixes that choice by the order in
which such stores were seen to land on a B200: within a warp the later store
instruction, for two lanes of one instruction the lower lane, across warps
the lower warp.  So the oracle is held to:

* every flip step on which all reference runs agree: the oracle's trace line
  (digests of triangles, neighbours, subsegments, status, active list and
  points) is the reference's, byte for byte;
* the first step on which the runs part: the oracle's live triangles equal
  the reference's as a set, i.e. the runs differ only in slot assignment;
* configurations whose runs all agree to the end: the oracle's output arrays
  are the reference's, byte for byte.
"""
import ctypes
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs
from oracle import oracle_py

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_outputs.json")
FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")

_doc = None


def load():
    global _doc
    if _doc is None:
        with open(GOLDEN) as f:
            _doc = json.load(f)
    return _doc


def digests(c):
    return {f: hashlib.sha256(np.ascontiguousarray(getattr(c, f)).tobytes()).hexdigest() for f in FIELDS}


def configs(size=None, consistent_only=False):
    out = []
    for name, case in load()["cases"].items():
        if size and case["size"] != size:
            continue
        for cfg in case["configs"]:
            if consistent_only and not cfg["self_consistent"]:
                continue
            out.append(pytest.param(name, cfg, id=f"{name}-{cfg['theta']}-p{cfg['policy']}-m{cfg['mode']}"))
    return out


_inputs = {}


def golden_input(name):
    case = load()["cases"][name]
    if name not in _inputs:
        c = eval(case["generator"], {"inputs": inputs})
        assert digests(c) == case["input"]["sha256"], "input generator drifted"
        _inputs[name] = c
    return _inputs[name]


def oracle_traced(name, cfg):
    """Oracle run with its flip-step trace; returns (output, trace lines)."""
    L = oracle_py.lib()
    L.gqm_oracle_trace.argtypes = [ctypes.c_char_p]
    gc2 = load()["device_goodcos2"][repr(cfg["theta"])]
    with tempfile.TemporaryDirectory() as d:
        tp = os.path.join(d, "trace.txt")
        L.gqm_oracle_trace(tp.encode())
        try:
            out, _ = oracle_py.refine(golden_input(name), cfg["theta"], cfg["policy"], cfg["mode"], goodcos2=gc2)
        finally:
            L.gqm_oracle_trace(None)
        lines = [l for l in open(tp) if l.startswith("F ")]
    return out, lines


def line_hash(line):
    return hashlib.sha256(line.strip().encode()).hexdigest()[:16]


@pytest.mark.parametrize("name,cfg", configs("small"))
def test_oracle_follows_reference_steps(name, cfg):
    out, lines = oracle_traced(name, cfg)
    tr = cfg["trace"]
    n = tr["agreed_steps"]
    assert len(lines) >= n
    mine = [line_hash(l) for l in lines[:n]]
    bad = next((i for i, (a, b) in enumerate(zip(mine, tr["line_hashes"])) if a != b), None)
    assert bad is None, f"oracle parts from every reference run at flip step {bad}"
    if tr["split_meshes"] and len(set(tr["split_meshes"])) == 1 and n < len(lines):
        # the runs part only in slot assignment: same live triangles
        assert lines[n].strip().rsplit("mesh=", 1)[1] == tr["split_meshes"][0]
    if cfg["self_consistent"]:
        assert len(lines) == tr["steps"][0]
        ref = cfg["runs"][0]
        assert (out.numberofpoints, out.numberoftriangles, out.numberofsegments) == (
            ref["points"], ref["triangles"], ref["segments"])
        assert digests(out) == ref["sha256"]


def test_fixture_has_self_consistent_configs_of_every_mode():
    combos = {(c["policy"], c["mode"]) for case in load()["cases"].values() for c in case["configs"]
              if c["self_consistent"]}
    assert combos == {(0, 0), (0, 1), (1, 0), (1, 1)}


# ---------------------------------------------------------------------------
# The reference as its project builds it (nvcc's default FMA contraction)
# ---------------------------------------------------------------------------
SPREAD = os.path.join(HERE, "golden", "reference_spread.json")


def _fma_entry(name, cfg):
    with open(SPREAD) as f:
        doc = json.load(f)
    for e in doc["cases"][name]:
        if (e["theta"], e["policy"], e["mode"]) == (cfg["theta"], cfg["policy"], cfg["mode"]):
            return e
    raise KeyError(name)


def fma_consistent_configs():
    """Configurations (CPU-sized, plus the 100,000-point hull-only one) on which
    every recorded run of the stock build gave the same output."""
    out = []
    for p in configs():
        name, cfg = p.values
        if load()["cases"][name]["size"] != "small" and name != "h100k":
            continue
        e = _fma_entry(name, cfg)
        if e["fma_self_consistent"] and e["fma_sha256"] == cfg["fma"]["sha256"]:
            out.append(p)
    return out


@pytest.mark.parametrize("name,cfg", fma_consistent_configs())
def test_contracted_oracle_matches_reference_as_built(name, cfg):
    """The oracle with the stock build's fused products (libgqm_oracle_fma.so)
    gives the stock build's output byte for byte."""
    gc2 = load()["device_goodcos2"][repr(cfg["theta"])]
    out, _ = oracle_py.refine(golden_input(name), cfg["theta"], cfg["policy"], cfg["mode"], goodcos2=gc2,
                              contracted=True)
    ref = cfg["fma"]
    assert (out.numberofpoints, out.numberoftriangles, out.numberofsegments) == (
        ref["points"], ref["triangles"], ref["segments"])
    assert digests(out) == ref["sha256"]


def test_contracted_configs_cover_every_mode():
    combos = {(p.values[1]["policy"], p.values[1]["mode"]) for p in fma_consistent_configs()}
    assert combos == {(0, 0), (0, 1), (1, 0), (1, 1)}
