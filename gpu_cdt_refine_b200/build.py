"""In-tree build of the native libraries (sm_100a CUDA and host C++).

    python -m gpu_cdt_refine_b200.build

libgqm_b200.so : refine.cu (kernels, driver, C ABI) + batch.cu (persistent
                 batched engine) + learned.cu (placement network training and
                 inference) + cdt_gpu.cu (CDT construction on the GPU) +
                 legacy.cpp (C++ drop-in)
libgqm_host.so : cdt_build.cpp + synth.cpp + certify.cpp

Every floating-point operation of the refiner is rounded on its own:
nvcc -fmad=false and gcc -ffp-contract=off, the same arithmetic as the
reference built with -fmad=false.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_host(force=False):
    out = os.path.join(HERE, "libgqm_host.so")
    srcs = [os.path.join(CSRC, f) for f in ("cdt_build.cpp", "synth.cpp", "certify.cpp")]
    deps = srcs + [os.path.join(CSRC, "predicates.h"), os.path.join(INC, "gqm_cdt.h")]
    if force or _stale(out, deps):
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off", "-I" + INC, "-o", out] + srcs)
    return out


def build_cuda(force=False, extra=None):
    out = os.path.join(HERE, "libgqm_b200.so")
    hdr = [os.path.join(INC, "gqm_refine.h"), os.path.join(INC, "gqm_triangulateio.h"),
           os.path.join(CSRC, "predicates.h"), os.path.join(CSRC, "host_copy.h")]
    refiner = [os.path.join(CSRC, f) for f in ("kernels.cuh", "gqm_device.cuh", "learned.cuh")]
    units = {  # translation unit -> the headers it includes
        "refine.cu": hdr + refiner,
        "batch.cu": hdr + refiner,
        "learned.cu": hdr + [os.path.join(CSRC, "learned.cuh")],
        "cdt_gpu.cu": [os.path.join(INC, "gqm_cdt.h"), os.path.join(CSRC, "predicates.h"),
                       os.path.join(CSRC, "host_copy.h")],
        "legacy.cpp": hdr,
    }
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler",
                    "-ffp-contract=off", "-I" + INC] + list(extra or [])
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    # stale translation units compile in parallel, then one link
    procs, objs = [], []
    for name, deps in units.items():
        src = os.path.join(CSRC, name)
        obj = os.path.join(objdir, name + ".o")
        objs.append(obj)
        if force or extra or _stale(obj, [src] + deps):
            cmd = [NVCC] + flags + ["-c", src, "-o", obj]
            print(" ".join(cmd), flush=True)
            procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("nvcc failed")
    if procs or _stale(out, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", out] + objs)
    return out


def build(force=False):
    build_host(force)
    build_cuda(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
