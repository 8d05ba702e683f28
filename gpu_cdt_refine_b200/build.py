"""In-tree build of the native libraries (sm_100a CUDA and host C++).

    python -m gpu_cdt_refine_b200.build

libgqm_b200.so : refine.cu (kernels, driver, C ABI) + batch.cu (persistent
                 batched engine, one-block small flip steps) + flipcl.cu
                 (small flip steps on a thread-block cluster) + learned.cu (placement network training and
                 inference) + cdt_gpu.cu (CDT construction on the GPU) +
                 legacy.cpp (C++ drop-in)
libgqm_b200_fma.so : the same with GQM_CONTRACTED set: the products that the
                 reference as its own project builds it (nvcc's default
                 contraction) fuses into an add or subtract are fused here
                 too, written out as fma() (gqm_madd in predicates.h)
libgqm_host.so : cdt_build.cpp + synth.cpp + certify.cpp + regions.cpp

Both are compiled without compiler contraction (nvcc -fmad=false, gcc
-ffp-contract=off), so the arithmetic is exactly the one the source writes: in
libgqm_b200.so every floating-point operation of the refiner is rounded on its
own (the reference built with -fmad=false), in libgqm_b200_fma.so the fused
products are the reference build's own.  The CPU oracle restates both
(oracle/_build/libgqm_oracle.so and libgqm_oracle_fma.so).
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
    srcs = [os.path.join(CSRC, f) for f in ("cdt_build.cpp", "synth.cpp", "certify.cpp", "regions.cpp")]
    deps = srcs + [os.path.join(CSRC, "predicates.h"), os.path.join(INC, "gqm_cdt.h")]
    if force or _stale(out, deps):
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off", "-I" + INC, "-o", out] + srcs)
    return out


# Refiner translation units: compiled once per arithmetic variant.
REFINER_UNITS = ("refine.cu", "batch.cu", "flipcl.cu")
# The arithmetic variants of the refiner:
#   "separate"   every product and sum rounded on its own: the reference built
#                with -fmad=false;
#   "contracted" GQM_CONTRACTED=1: fma() exactly where the reference as its
#                project builds it (no -fmad option, so nvcc contracts) fuses.
VARIANTS = {"separate": ("libgqm_b200.so", "-fmad=false", "_build"),
            "contracted": ("libgqm_b200_fma.so", "-fmad=false", os.path.join("_build", "fma"))}


def _cuda_jobs(force=False, extra=None, variant="separate"):
    """(library path, object paths, compile commands of the stale objects)."""
    lib, fmad, objsub = VARIANTS[variant]
    out = os.path.join(HERE, lib)
    hdr = [os.path.join(INC, "gqm_refine.h"), os.path.join(INC, "gqm_triangulateio.h"),
           os.path.join(CSRC, "predicates.h"), os.path.join(CSRC, "host_copy.h")]
    refiner = [os.path.join(CSRC, f) for f in ("kernels.cuh", "gqm_device.cuh", "learned.cuh")]
    units = {  # translation unit -> (the headers it includes, its own flags)
        "refine.cu": (hdr + refiner, []),
        "batch.cu": (hdr + refiner, []),
        # phases on several SMs of a cluster: global loads are cached in L2 only
        "flipcl.cu": (hdr + refiner, ["-Xptxas", "-dlcm=cg"]),
        "learned.cu": (hdr + [os.path.join(CSRC, "learned.cuh")], []),
        "cdt_gpu.cu": ([os.path.join(INC, "gqm_cdt.h"), os.path.join(CSRC, "predicates.h"),
                        os.path.join(CSRC, "host_copy.h")], []),
        "legacy.cpp": (hdr, []),
    }
    base = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                   "-I" + INC] + list(extra or [])
    objdir = os.path.join(HERE, "_build")
    vdir = os.path.join(HERE, objsub)
    os.makedirs(vdir, exist_ok=True)
    objs, cmds = [], []
    for name, (deps, own) in units.items():
        src = os.path.join(CSRC, name)
        mine = name in REFINER_UNITS
        obj = os.path.join(vdir if mine else objdir, name + ".o")
        objs.append(obj)
        # the units outside the refiner are shared by the variants (always
        # -fmad=false) and compiled by the "separate" variant's jobs only
        if (mine or variant == "separate") and (force or extra or _stale(obj, [src] + deps)):
            flags = base + [fmad if mine else "-fmad=false"] + own
            if mine and variant == "contracted":
                flags = flags + ["-DGQM_CONTRACTED=1"]
            cmds.append([NVCC] + flags + ["-c", src, "-o", obj])
    return out, objs, cmds


def build_cuda(force=False, extra=None, variants=("separate", "contracted")):
    """Compile the stale objects of every variant in parallel, then link each
    library whose objects changed."""
    jobs = [_cuda_jobs(force, extra, v) for v in variants]
    procs = []
    for _, _, cmds in jobs:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
            procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("nvcc failed")
    outs = []
    for out, objs, _ in jobs:
        if procs or _stale(out, objs):
            _run([NVCC] + ARCH + ["-shared", "-o", out] + objs)
        outs.append(out)
    return outs[0]


def build(force=False):
    build_host(force)
    build_cuda(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
