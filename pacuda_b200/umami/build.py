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


def stale(out: str, inputs) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(x) > t for x in inputs)


def build(provider: str, out: str, runner_dir: str = PKG) -> str:
    provider = os.path.abspath(provider)
    cmd = [NVCC, "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off", "-shared",
           "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.dirname(provider),
           f'-DUMAMI_PROVIDER_HEADER="{os.path.basename(provider)}"',
           "-o", out] + SOURCES + ["-L", runner_dir, "-lrecurrence", f"-Xlinker=-rpath,{runner_dir}"]
    subprocess.run(cmd, check=True)
    return out


PP3J = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"]


def pp3j_spec():
    """The p p -> 3 jets subprocess families as one UMAMI subprocess: channel 0, flavour k = family
    k (its plan with the identity permutation)."""
    return {"particles": 5, "masses": [0.0] * 5, "colors": 1,
            "processes": [{"key": k, "helicities": 32, "parameters": [("aS", 0.118, 0.0, False, True)]}
                          for k in PP3J],
            "channels": [[[{"process": i, "colour": "lc", "permutation": [0, 1, 2, 3, 4], "factor": 1.0}]
                          for i in range(len(PP3J))]],
            "has_alpha_s": True, "has_color_flow": False}


def pp3j_library() -> str:
    """The UMAMI library of the p p -> 3 jets families, built in-tree (pacuda_b200/umami/_build)
    when missing or older than its sources."""
    from . import provider

    d = os.path.join(HERE, "_build")
    os.makedirs(d, exist_ok=True)
    hdr = os.path.join(d, "provider_pp3j.h")
    text = provider.header(pp3j_spec())
    if not os.path.exists(hdr) or open(hdr).read() != text:
        with open(hdr, "w") as f:
            f.write(text)
    out = os.path.join(d, "libumami_pp3j.so")
    deps = SOURCES + [hdr, os.path.join(HERE, "pacuda_reader.h"), os.path.join(PKG, "librecurrence.so"),
                      os.path.join(ROOT, "include", "umami.h"), os.path.join(ROOT, "include", "umami_provider.h"),
                      os.path.join(ROOT, "include", "pacuda_b200.h")]
    if stale(out, deps):
        build(hdr, out)
    return out


if __name__ == "__main__":
    build(sys.argv[1], sys.argv[2])
