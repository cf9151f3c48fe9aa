"""Builds a subprocess's UMAMI library (pacuda_b200/umami/umami_b200.cu) against its provider
header and this package's librecurrence.so, as the reference builds its own (umami/build.sh).

    python -m pacuda_b200.umami.build PROVIDER.h OUT.so
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = [os.path.join(HERE, "umami_b200.cu"), os.path.join(HERE, "pacuda_reader.cpp")]


def build(provider: str, out: str, runner_dir: str = PKG) -> str:
    provider = os.path.abspath(provider)
    cmd = [NVCC, "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off", "-shared",
           "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.dirname(provider),
           f'-DUMAMI_PROVIDER_HEADER="{os.path.basename(provider)}"',
           "-o", out] + SOURCES + ["-L", runner_dir, "-lrecurrence", f"-Xlinker=-rpath,{runner_dir}"]
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    build(sys.argv[1], sys.argv[2])
