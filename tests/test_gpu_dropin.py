"""Drop-in check of GPU_Refine_Quality: the reference's own driver code
(oracle/ref_driver.cu, compiled against the reference's GPU_Refine/refine.h)
linked to this library instead of the reference's refine.cu
(oracle/_ref/gqm_dropin_run, built by oracle/Makefile).  Through the
reference's header, structures and calling convention, the C++ entry point
returns the same refined CDT as the C ABI, byte for byte, and hands back
arrays the caller releases with delete[] (the driver does)."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from gpu_cdt_refine_b200 import cdtio, inputs, refine

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "gqm_dropin_run")


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in driver (make -C oracle ref) not present")
@pytest.mark.parametrize("policy,mode", [(1, 1), (0, 0)])
def test_reference_driver_links_and_matches(gpu, policy, mode):
    cdt = inputs.clustered(seed=371, n=20_000, nseg=1000)
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        cdtio.write_cdt(src, cdt)
        p = subprocess.run([DROPIN, src, dst, "20.0", str(policy), str(mode), "2"], capture_output=True,
                           text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-400:]
        info = json.loads([l for l in p.stderr.splitlines() if l.startswith("GQMREF ")][0][7:])
        got = cdtio.read_cdt(dst)
    want, _ = refine.refine(cdt, 20.0, policy, mode)
    assert (info["points"], info["triangles"], info["segments"]) == (
        want.numberofpoints, want.numberoftriangles, want.numberofsegments)
    for f in ("pointlist", "trianglelist", "neighborlist", "segmentlist"):
        assert np.array_equal(getattr(got, f), getattr(want, f)), f
