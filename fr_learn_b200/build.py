"""Builds fr_learn_b200/libfrgpu.so in-tree for sm_100a.

    python -m fr_learn_b200.build            # incremental
    python -m fr_learn_b200.build --force

Host set-up code (csrc/setup.cpp) is compiled by g++ -O2 without -march so
its floating-point arithmetic matches a plain x86-64 build of the reference;
the CUDA sources are compiled by nvcc for sm_100a only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfrgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC"]

CU_SOURCES = ["frgpu.cu", "integrals.cu", "stage_2d_f64.cu", "stage_2d_f32.cu", "stage_3d_f64.cu", "stage_3d_f32.cu",
              "adjoint_2d.cu", "adjoint_3d.cu", "opgemm.cu", "metrics.cu"]
# The FP32 arithmetic of the mixed mode uses the hardware's approximate
# single-precision divide and square root (within 2 ulp); FP64 arithmetic is
# unaffected by these flags, so the FP64 units stay exact.
UNIT_FLAGS = {u: ["-prec-div=false", "-prec-sqrt=false"] for u in ("stage_2d_f32.cu", "stage_3d_f32.cu")}
CXX_SOURCES = ["setup.cpp", "restart.cpp", "gmsh.cpp"]
HEADERS = ["kernels.cuh", "kernels_tma.cuh", "kernels_visc_tma.cuh", "adjoint.cuh", "adjoint_visc.cuh", "adjoint_impl.cuh", "dual.cuh", "optab_upload.cuh",
           "physics.cuh", "setup.h", "dispatch.h", "stage_impl.cuh"]


def _nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else shutil.which("nvcc")


def _cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no g++ found")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {os.path.basename(cmd[-1])}")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "frgpu.h")]
    objs = []
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            _run([_cxx()] + CXX_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            jobs.append([_nvcc()] + NVCC_FLAGS + UNIT_FLAGS.get(src, []) + (["-Xptxas", "-v"] if verbose else [])
                        + ["-c", s, "-o", o])
        objs.append(o)
    # the kernel units are independent: compile them in parallel
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in ex.map(_run, jobs):
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _newer(LIB, objs):
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
