"""Build recipe for the native parts of caustic_b200.

``libcausticot.so`` (the C ABI in include/causticot.h) is compiled in-tree
for sm_100a with nvcc; ``caustic_GPU`` (the process + file shim of the
reference executable) links against it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libcausticot.so")
CLI = os.path.join(PKG, "caustic_GPU")
CU_SOURCES = ["cot_cells.cu", "cot_solver.cu", "cot_capi.cu", "cot_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, "cot_common.cuh"), os.path.join(ROOT, "include", "causticot.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-shared", "-o", LIB, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "caustic_gpu_main.cpp")
    if not os.path.exists(src):
        return ""
    if not force and not _stale(CLI, [src, LIB, os.path.join(CSRC, "json_min.hpp")]):
        return CLI
    cmd = ["g++", "-O2", "-std=c++17", "-o", CLI, src, "-I", os.path.join(ROOT, "include"),
           "-L", PKG, "-lcausticot", f"-Wl,-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    return CLI


def build(force: bool = False, verbose: bool = False):
    build_lib(force, verbose)
    build_cli(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
