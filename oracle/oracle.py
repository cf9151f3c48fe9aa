"""Python access to the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY: imported by tests/,
by __graft_entry__.smoke() and by bench.py's CPU-baseline leg; never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build():
    """Compile liboracle.so (and, when the reference sources are mounted, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.oracle_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        for name in ("oracle_reduce", "oracle_reduce_resolved", "oracle_reduce_sample"):
            getattr(_lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        _lib.oracle_sources.argtypes = [C.c_void_p] * 3 + [C.c_uint32] + [C.c_void_p] * 2
        _lib.oracle_decode.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p, C.c_uint32]
    return _lib


def run(call_args, kernel=1, sort=True, threads=0):
    """oracle_run on a `pacuda_b200.abi.CallArgs` (its arrays are the arena, updated in place)."""
    return lib().oracle_run(C.addressof(call_args.struct), int(kernel), 1 if sort else 0, int(threads))


def reduce_resolved(r, are, aim, stride):
    return lib().oracle_reduce_resolved(C.addressof(r), are.ctypes.data, aim.ctypes.data, stride)


def reduce(r, are, aim, stride):
    return lib().oracle_reduce(C.addressof(r), are.ctypes.data, aim.ctypes.data, stride)


def reduce_sample(r, are, aim, stride):
    return lib().oracle_reduce_sample(C.addressof(r), are.ctypes.data, aim.ctypes.data, stride)


def sources(codes, masses, momenta):
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    masses = np.ascontiguousarray(masses, dtype=np.float64)
    momenta = np.ascontiguousarray(momenta, dtype=np.float64)
    n = len(codes)
    re, im = np.zeros(4 * n), np.zeros(4 * n)
    assert lib().oracle_sources(codes.ctypes.data, masses.ctypes.data, momenta.ctypes.data, n,
                                re.ctypes.data, im.ctypes.data) == 0
    return re.reshape(n, 4) + 1j * im.reshape(n, 4)


def decode(words, width, sort=True):
    words = np.ascontiguousarray(words, dtype=np.uint64)
    width = np.ascontiguousarray(width, dtype=np.uint8)
    n = lib().oracle_decode(words.ctypes.data, len(words), width.ctypes.data, 1 if sort else 0, None, 0)
    if n < 0:
        raise ValueError("malformed plan")
    out = np.zeros(9 * max(n, 1), dtype=np.uint32)
    lib().oracle_decode(words.ctypes.data, len(words), width.ctypes.data, 1 if sort else 0, out.ctypes.data, n)
    return out[: 9 * n].reshape(n, 9)


def evaluate(template, momenta, kernel=1, threads=0, sort=True):
    """Every amplitude of `template` at point-major momenta [point][leg][4]: an array
    [amplitude plane][point] of complex values, and the resolved outputs [point][output]."""
    from pacuda_b200 import abi, phase_space

    points = momenta.shape[0]
    ext = phase_space.source_major(momenta)
    args = template.call(ext, points)
    status = run(args, kernel=kernel, threads=threads, sort=sort)
    if status != 0:
        raise RuntimeError(f"oracle_run returned {status}")
    are, aim = args.are, args.aim
    amps = (are + 1j * aim).reshape(template.amplitude_planes, points)
    out = np.zeros(points * template.outputs)
    r, keep = abi.reduce_resolved_args(template.planes, template.weights, template.offsets, out, points, 1,
                                       template.outputs, abi.OUTPUT_ZERO)
    assert reduce_resolved(r, are, aim, points) == 0
    return amps, out.reshape(points, template.outputs)
