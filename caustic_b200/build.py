"""Build recipe for the native parts of caustic_b200.

``libcausticot.so`` (the C ABI in include/causticot.h) is compiled in-tree
for sm_100a with nvcc; ``caustic_GPU`` (the process + file shim of the
reference executable) links against it.  ``libcausticws.so`` (the warm-start
network's kernels, include/causticws.h) is built apart because its
tensor-core GEMMs come from the CUTLASS sm100 templates, which take a while
to compile.
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
CU_SOURCES = ["cot_cells.cu", "cot_solver.cu", "cot_capi.cu", "cot_noalloc.cu", "cot_newton.cu", "cot_build.cu"]
WS_LIB = os.path.join(PKG, "libcausticws.so")
WS_SOURCES = ["wsn.cu", "ws_predict.cu"]
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
    deps = srcs + [os.path.join(CSRC, "cot_common.cuh"), os.path.join(CSRC, "cot_edge.cuh"),
                   os.path.join(ROOT, "include", "causticot.h")]
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


def cutlass_dirs() -> list:
    """Include directories of a CUTLASS tree with the sm100 collectives
    (CUTLASS_DIR, else the copies vendored by installed packages)."""
    cands = []
    if os.environ.get("CUTLASS_DIR"):
        cands.append(os.environ["CUTLASS_DIR"])
    try:
        import site

        for sp in site.getsitepackages():
            cands.append(os.path.join(sp, "flashinfer", "data", "cutlass"))
            cands.append(os.path.join(sp, "tilelang", "3rdparty", "cutlass"))
    except Exception:
        pass
    for c in cands:
        inc = os.path.join(c, "include")
        if os.path.exists(os.path.join(inc, "cutlass", "gemm", "collective", "builders", "sm100_umma_builder.inl")):
            return [inc, os.path.join(c, "tools", "util", "include")]
    raise RuntimeError("no CUTLASS tree with the sm100 collectives found (set CUTLASS_DIR)")


def build_ws(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in WS_SOURCES]
    deps = srcs + [os.path.join(ROOT, "include", "causticws.h")]
    if not force and not _stale(WS_LIB, deps):
        return WS_LIB
    inc = []
    for d in cutlass_dirs():
        inc += ["-I", d]
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-diag-suppress", "20012",
           *inc, "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared", "-o", WS_LIB, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return WS_LIB


def build(force: bool = False, verbose: bool = False):
    build_lib(force, verbose)
    build_cli(force)
    build_ws(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
