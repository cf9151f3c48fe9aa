"""Builds the runner library pacuda_b200/librecurrence.so in the source tree (nvcc, sm_100a).

The library is the product: the C ABI of include/pacman_recurrence.h. It is compiled with
-fmad=false so that no multiply-add is contracted (the f64 kernel's arithmetic is the
reference's, operation by operation) and linked against the static CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librecurrence.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["runner.cu", "batch.cu", "program.cpp", "schedule.cpp", "tiled_host.cu", "peak.cu"]
FLAGS = ["-O3", "-std=c++17", "-fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
         "-gencode", "arch=compute_100a,code=sm_100a", "-Xptxas", "-warn-spills"]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "pacman_recurrence.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    cmd = [NVCC] + FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
