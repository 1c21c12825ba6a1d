"""Builds libchronos_b200.so in-tree with nvcc for sm_100a (plus the host C++
with g++/OpenMP).  Run `python -m chronoslab_b200.build` or call build().

Objects go to chronoslab_b200/_build/; the shared library to
chronoslab_b200/libchronos_b200.so (both git-ignored; the .so travels with the
tree to the GPU machine).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchronos_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The system g++ carries libgomp's link spec (a CXX from the environment may not).
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

CU_SOURCES = ["setup_kernels.cu", "hier.cu", "block.cu", "batch.cu", "group.cu", "capi.cu",
              "coarsen_gpu.cu", "gmres.cu", "bamg_gpu.cu", "emin_gpu.cu"]
# per-file flags: the GPU BAMG reproduces the host restatement (built with
# -ffp-contract=off) bit for bit, so its products and sums are not fused
CU_EXTRA = {"bamg_gpu.cu": ["-fmad=false"]}
CPP_SOURCES = ["host/params.cpp", "host/coarsen.cpp", "host/bamg.cpp", "host/fsai_pattern.cpp",
               "host/formats.cpp", "host/emin.cpp"]
HEADERS = ["common.cuh", "errors.h", "internal.h", "hier.h", "group.h", "spmv.cuh", "host/host.h"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                        "-ccbin", CXX, "-Xcompiler", "-fPIC,-fopenmp", "-Xptxas",
                        "-warn-spills"]
CXX_FLAGS = ["-O3", "-fPIC", "-fopenmp", "-std=c++17", "-ffp-contract=off",
             f"-I{CUDA_HOME}/include"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "chronos_b200.h")]
    tasks, objs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            tasks.append([NVCC] + NVCC_FLAGS + CU_EXTRA.get(src, []) + ["-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            tasks.append([CXX] + CXX_FLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for out in ex.map(_run, tasks):
            if verbose and out.strip():
                print(out)
    if tasks or not os.path.exists(LIB):
        out = _run([NVCC] + GENCODE + ["-shared", "-ccbin", CXX, "-o", LIB] + objs +
                   ["-Xcompiler", "-fopenmp", "-lgomp"])
        if verbose and out.strip():
            print(out)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
