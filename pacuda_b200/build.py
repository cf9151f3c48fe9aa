"""Builds the libraries in the source tree (nvcc, sm_100a).

* pacuda_b200/librecurrence.so: the runner, the C ABI of include/pacman_recurrence.h and the
  batched API of include/pacuda_b200.h. Compiled with -fmad=false so that no multiply-add is
  contracted (the f64 kernel's arithmetic is the reference's, operation by operation) and linked
  against the static CUDA runtime.
* pacuda_b200/libsurrogate.so: the surrogate network (include/pacuda_surrogate.h) and the
  two-stage unweighting kernels; free to contract multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(HERE, "..", "include")
LIB = os.path.join(HERE, "librecurrence.so")
SG_LIB = os.path.join(HERE, "libsurrogate.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["runner.cu", "batch.cu", "program.cpp", "schedule.cpp", "tiled_host.cu", "peak.cu", "stability.cu"]
SG_SOURCES = ["surrogate.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
         "-Xptxas", "-warn-spills"] + ARCH
SG_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
            "-Xptxas", "-warn-spills"] + ARCH

RUNNER_DEPS = ["runner.cu", "batch.cu", "program.cpp", "program.h", "schedule.cpp", "schedule.h", "tiled_host.cu",
               "tiled_host.h", "peak.cu", "arith.cuh", "executor.cuh", "tiled.cuh", "tiled_fma.cu", "stability.cu"]
SG_DEPS = ["surrogate.cu", "umma.cuh"]


def _stale(target, deps, headers):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    paths = [os.path.join(CSRC, f) for f in deps] + [os.path.join(INCLUDE, h) for h in headers]
    return any(os.path.getmtime(d) > t for d in paths if os.path.exists(d))


def stale():
    return _stale(LIB, RUNNER_DEPS, ["pacman_recurrence.h", "pacuda_b200.h"]) or \
        _stale(SG_LIB, SG_DEPS, ["pacuda_surrogate.h"])


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False):
    if force or _stale(LIB, RUNNER_DEPS, ["pacman_recurrence.h", "pacuda_b200.h"]):
        # the f64 kind with contracted multiply-adds: the same executor compiled with -fmad=true
        obj = os.path.join(CSRC, "..", "tiled_fma.o")
        _run([NVCC] + [f if f != "-fmad=false" else "-fmad=true" for f in FLAGS if f not in ("-shared",)] +
             ["-c", "-o", obj, os.path.join(CSRC, "tiled_fma.cu")], verbose)
        _run([NVCC] + FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES] + [obj], verbose)
        os.unlink(obj)
    if force or _stale(SG_LIB, SG_DEPS, ["pacuda_surrogate.h"]):
        _run([NVCC] + SG_FLAGS + ["-o", SG_LIB] + [os.path.join(CSRC, s) for s in SG_SOURCES], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
