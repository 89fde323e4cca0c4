"""Build recipe: compiles csrc/ for sm_100a into an in-tree shared library
(librism3d_b200.so, next to this file) and the drop-in CLI (bin/rism3d-b200).
Cross-compiles without a GPU; objects go to csrc/_build/."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
TOP = os.path.dirname(PKG)                       # 3d-rism-cuda_b200/
ROOT = os.path.dirname(TOP)                      # repository root
CSRC = os.path.join(TOP, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(PKG, "librism3d_b200.so")
CLI = os.path.join(TOP, "bin", "rism3d-b200")
CLI1D = os.path.join(TOP, "bin", "rism1d-b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["potential.cu", "solver.cu", "observe.cu", "adjoint.cu", "batch.cu",
           "noalloc.cu", "rmdft.cu", "capi.cpp", "io.cpp", "xrism1d.cpp"]


def _ccbin():
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _flags():
    return (_ccbin() + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                               "-I" + os.path.join(ROOT, "include"), "-I" + CSRC])


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose=False):
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src + ".o")
    hdrs = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "rism3d_b200.h"))
    if _newer(o, [s] + hdrs):
        cmd = [NVCC] + _flags() + ["-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
    return o


def build(verbose=False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _newer(LIB, objs):
        subprocess.check_call([NVCC] + _ccbin() + ARCH + ["-shared", "-o", LIB] + objs +
                              ["-lcufft", "-lcudart"])
    for exe, src in ((CLI, "cli.cpp"), (CLI1D, "cli1d.cpp")):
        cli_src = os.path.join(CSRC, src)
        if _newer(exe, [cli_src, LIB]):
            subprocess.check_call([NVCC] + _ccbin() + ["-O2", "-std=c++17",
                                   "-I" + os.path.join(ROOT, "include"), cli_src, "-o", exe,
                                   "-L" + PKG, "-lrism3d_b200",
                                   "-Xlinker", "-rpath=$ORIGIN/../rism3d_b200"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
