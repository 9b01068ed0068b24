"""In-tree build of the tspeed_b200 shared library for sm_100a.

    python -m tspeed_b200.build            # builds tspeed_b200/libtspeed_b200.so
    python -m tspeed_b200.build --checked  # also tspeed_b200/libtspeed_b200_checked.so

The checked library is the same code compiled with TSP_CHECKED: the step
kernels range-check every gather index they read on the device (see
tsp_checked_build in include/tspeed_b200.h); tspeed_b200.capi loads it when
TSP_CHECKED=1 is set in the environment.

nvcc cross-compiles without a GPU. The library is a plain C-ABI .so (no
torch types), loaded by ctypes (tspeed_b200.capi) or linked by C/C++ hosts.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtspeed_b200.so")
LIB_CHECKED = os.path.join(HERE, "libtspeed_b200_checked.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
SOURCES = ["tsp_host.cpp", "tsp_capi.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False, checked: bool = False) -> str:
    """Builds the library (checked=True: the TSP_CHECKED variant) and returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "tspeed_b200.h"))
    lib = LIB_CHECKED if checked else LIB
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        # The host C++ object is shared; the CUDA object differs by TSP_CHECKED.
        tag = ".checked" if checked and src.endswith(".cu") else ""
        obj = os.path.join(BUILD, src + tag + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
            if tag:
                cmd.append("-DTSP_CHECKED")
            if ptxas_verbose and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
    if "--checked" in sys.argv:
        print(build(verbose=True, force="--force" in sys.argv, checked=True))
