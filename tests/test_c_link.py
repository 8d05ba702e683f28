"""The headers are usable from plain C and C++: programs compiled against
include/gqm_refine.h and include/gqm_triangulateio.h link libgqm_b200.so,
and on a machine without a GPU they get status codes back (the C ABI) or an
empty result with a message (the reference's C++ entry point), never an exit
of the process."""
import os
import subprocess

import pytest

from gpu_cdt_refine_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(_native.CUDA_LIB)

C_PROGRAM = r"""
#include <stdio.h>
#include "gqm_refine.h"
int main(void) {
  /* a unit square split into two triangles, its four sides as segments */
  double pts[8] = {0, 0, 1, 0, 1, 1, 0, 1};
  int tri[6] = {0, 1, 2, 0, 2, 3};
  int nbr[6] = {-1, 1, -1, -1, -1, 0};
  int seg[8] = {0, 1, 1, 2, 2, 3, 3, 0};
  gqm_cdt_in in = {4, pts, 2, tri, nbr, 4, seg};
  gqm_cdt_out out;
  gqm_options opt;
  gqm_default_options(&opt);
  if (opt.theta != 20.0 || opt.insert_policy != GQM_OFFCENTER || opt.mode != GQM_RUPPERT) return 2;
  opt.theta = 0.0;
  int bad = gqm_refine(&in, &out, &opt, NULL);
  opt.theta = 20.0;
  int rc = gqm_refine(&in, &out, &opt, NULL);
  printf("%d %d %s\n", bad, rc, gqm_status_string(rc));
  if (rc == 0) gqm_free_result(&out);
  return 0;
}
"""

CXX_PROGRAM = r"""
#include <cstdio>
#include "gqm_triangulateio.h"
int main() {
  double pts[8] = {0, 0, 1, 0, 1, 1, 0, 1};
  int tri[6] = {0, 1, 2, 0, 2, 3};
  int nbr[6] = {-1, 1, -1, -1, -1, 0};
  int seg[8] = {0, 1, 1, 2, 2, 3, 3, 0};
  triangulateio in = {}, out = {};
  in.pointlist = pts; in.numberofpoints = 4;
  in.trianglelist = tri; in.neighborlist = nbr; in.numberoftriangles = 2; in.numberofcorners = 3;
  in.segmentlist = seg; in.numberofsegments = 4;
  GPU_Refine_Quality(&in, &out, 20.0, Offcenter, Connected, 1, -1, nullptr, nullptr);
  std::printf("returned %d %d %d\n", out.numberofpoints, out.numberoftriangles, out.numberofsegments);
  delete[] out.pointlist;
  delete[] out.trianglelist;
  delete[] out.neighborlist;
  delete[] out.segmentlist;
  return 0;
}
"""


def _build_and_run(tmp_path, name, source, compiler):
    src = tmp_path / name
    src.write_text(source)
    exe = tmp_path / (name + ".bin")
    subprocess.check_call([compiler, "-O1", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                           "-L" + LIBDIR, "-lgqm_b200", "-Wl,-rpath," + LIBDIR])
    return subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)


@pytest.fixture(scope="module")
def no_gpu():
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("checks the behaviour without a CUDA device")


def test_c_program_gets_status_codes(tmp_path, no_gpu):
    r = _build_and_run(tmp_path, "use_abi.c", C_PROGRAM, "gcc")
    assert r.returncode == 0, r.stderr
    bad, rc, _ = r.stdout.split(maxsplit=2)
    assert int(bad) == -1        # GQM_ERR_ARGUMENT: theta 0 rejected on the host
    assert int(rc) == -11        # GQM_ERR_NO_DEVICE


def test_cxx_drop_in_returns_empty_result_instead_of_exiting(tmp_path, no_gpu):
    r = _build_and_run(tmp_path, "use_dropin.cpp", CXX_PROGRAM, "g++")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "returned 0 0 0"
    assert "GPU_Refine_Quality" in r.stderr
