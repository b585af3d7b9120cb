"""Build libflowmap_sm100.so (the C-ABI CUDA library) in-tree with nvcc.

Usage: ``python differentiable-flowmap_b200/build.py [--verbose-ptxas]``.
The library is compiled for sm_100a only; nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libflowmap_sm100.so")
SOURCES = ["fm_flowmap.cu", "fm_mgpcg.cu", "fm_util.cu", "fm_stencil.cu", "fm_vortex.cu", "fm_force.cu", "fm_solid.cu",
           "fm_adjoint.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "flowmap_sm100.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *ARCH]
    if ptxas_verbose:
        flags += ["-Xptxas", "-v"]
    procs = []
    for src in SOURCES:  # translation units compile in parallel
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        procs.append(subprocess.Popen([nvcc, *flags, "-c", os.path.join(CSRC, src), "-o", obj]))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    tmp = LIB + ".tmp"
    # static CUDA runtime: the library does not depend on the version of
    # libcudart that the host process (e.g. torch) happens to have loaded
    subprocess.run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, ptxas_verbose="--verbose-ptxas" in sys.argv)
    print(LIB)
