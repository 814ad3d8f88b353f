"""Builds libmenos_b200.so in-tree: host C++ (g++) + sm_100a CUDA (nvcc).

    python -m menos_b200.build

Flags that carry the bitwise contract: host code -ffp-contract=off (no a*b+c
contraction, as the reference's CPU kernels, src/kernels/CMakeLists.txt:19);
device code -fmad=false (as the reference's CUDA kernels,
src/kernels/cuda/CMakeLists.txt:66) on top of the explicit __dmul_rn /
__dadd_rn intrinsics.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "build", "obj")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libmenos_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX_FLAGS = ["-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
             f"-I{CUDA_HOME}/include", f"-I{os.path.join(ROOT, 'include')}"]
NVCC_FLAGS = ["-std=c++20", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"] + ARCH


def _sources():
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    return cpp, cu


def _newer(src_paths, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {cmd[-1]}")
    return r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source whose inputs changed and links the library.
    Returns the library path."""
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    cpp, cu = _sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "mb2.h"))
    jobs, objs = [], []
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj):
            jobs.append([CXX] + CXX_FLAGS + ["-c", "-o", obj, src])
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _newer([src] + headers, obj) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", "-o", obj, src])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_compile, jobs):
            if verbose and out:
                sys.stderr.write(out)
    if jobs or not os.path.exists(LIB):
        cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-cudart", "static", "-lpthread"]
        _compile(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
