"""The sm_100a refiner against the reference's own runs: wherever every run of
the reference produced the same output (all golden configurations whose runs
agree, including those too large for the CPU oracle), the refiner's output
is that output, byte for byte."""
import pytest

from gpu_cdt_refine_b200 import refine
from test_golden import configs, digests, golden_input, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,cfg", configs(consistent_only=True))
def test_gpu_matches_reference(gpu, name, cfg):
    got, st = refine.refine(golden_input(name), cfg["theta"], cfg["policy"], cfg["mode"])
    assert st["goodcos2"] == load()["device_goodcos2"][repr(cfg["theta"])]
    ref = cfg["runs"][0]
    assert (got.numberofpoints, got.numberoftriangles, got.numberofsegments) == (
        ref["points"], ref["triangles"], ref["segments"])
    assert digests(got) == ref["sha256"]
