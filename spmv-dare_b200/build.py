"""Build recipe of libspmv_b200.so (sm_100a), in-tree.

    python spmv-dare_b200/build.py            # incremental
    python spmv-dare_b200/build.py --clean

CUDA sources are compiled with nvcc for sm_100a only; the host generator (artgen.c) with
gcc using the reference's optimisation flags (-O3, an AVX2+FMA x86-64 target) so its
floating-point expressions are contracted exactly as in the reference build.  The shared
library lands in spmv-dare_b200/lib/ (git-ignored, shipped with the tree).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libspmv_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
if not os.path.exists(NVCC):
    NVCC = shutil.which("nvcc") or NVCC
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I" + INCLUDE, "-I" + CSRC,
                     "--expt-relaxed-constexpr", "-diag-suppress", "177"]
CUDA_INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(NVCC))), "include")
GCC_FLAGS = ["-O3", "-march=x86-64-v3", "-fPIC", "-fopenmp", "-std=gnu11", "-Wall", "-Wno-unused-result",
             "-I" + CUDA_INCLUDE]

CU_SOURCES = ["primitives.cu", "convert.cu", "spmv_kernels.cu", "warp_kernels.cu", "div.cu", "fp32.cu", "batch.cu", "select.cu",
              "mtx.cu", "pack.cu", "sym.cu", "gen.cu", "api.cu"]
C_SOURCES = ["artgen.c", "mtx_parse.c", "hostcopy.c"]
HEADERS = ["common.cuh", "primitives.cuh", "internal.h", "mtx_parse.h", "hostcopy.h"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list if os.path.exists(s))


def _run(cmd):
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + p.stdout)
    return p.stdout


def build(verbose=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "spmv_b200.h")]
    steps = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj):
            steps.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for s in C_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj):
            steps.append(["gcc"] + GCC_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for out in ex.map(_run, steps):
            if verbose and out.strip():
                print(out)
    if steps or _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lcudart", "-lm"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    if a.clean:
        shutil.rmtree(OBJ, ignore_errors=True)
        if os.path.exists(LIB):
            os.remove(LIB)
    print(build(verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
