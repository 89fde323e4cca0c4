"""Build recipe for the oracle -- TEST INFRASTRUCTURE.

* ``liboracle_rism3d.so``: the CPU FP64 OpenMP restatement (own sources).
* ``_ref/3drism-cuda``: the reference executable compiled from its own
  sources where they lie (``ref.mk``); only when the reference tree exists.
Both outputs are git-ignored and travel to the GPU box with the snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle_rism3d.so")
# The reference checkout: $RISM3D_REFERENCE, by default where the build
# container mounts it.
REFERENCE = os.environ.get("RISM3D_REFERENCE", "/root/reference")
REF_SRC = os.path.join(REFERENCE, "src-cuda")
REF_BIN = os.path.join(HERE, "_ref", "3drism-cuda")


def host_cxx() -> str:
    # The image's exported CXX wrapper cannot link OpenMP; prefer the system g++.
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "rism3d_oracle.cpp")
    hdr = os.path.join(HERE, "rism3d_oracle.h")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cmd = [host_cxx(), "-O3", "-march=x86-64-v2", "-fopenmp", "-std=c++17",
           "-shared", "-fPIC", src, "-o", LIB]
    subprocess.check_call(cmd)
    return LIB


def build_reference() -> str | None:
    """Compile the reference CUDA executable for sm_100a (checker + reference arm)."""
    if not os.path.isdir(REF_SRC):
        return REF_BIN if os.path.exists(REF_BIN) else None
    jobs = str(max(1, os.cpu_count() or 1))
    subprocess.check_call(["make", "-s", "-f", os.path.join(HERE, "ref.mk"),
                           "REF=" + REF_SRC, "OUT=" + os.path.join(HERE, "_ref"),
                           "-j" + jobs])
    return REF_BIN


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_reference())
