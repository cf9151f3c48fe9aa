"""Python access to a recurrence runner library through its C ABI (ctypes).

`Runner(path)` binds any library with the pacman_recurrence v1 ABI: this package's
librecurrence.so (the default) or the reference runner built from its sources. The product path
fails loudly when the library is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "librecurrence.so")


class RunnerError(RuntimeError):
    pass


class Runner:
    def __init__(self, path=None, kernel=None, block=0, no_sort=False, stats=False, executor=None):
        path = path or DEFAULT_LIB
        if not os.path.exists(path):
            raise RunnerError(f"{path}: the runner library is not built (python -m pacuda_b200.build)")
        self.path = path
        self.lib = C.CDLL(path)
        L = self.lib
        for name in ("pacman_recurrence_v1_run", "pacman_recurrence_v1_reduce", "pacman_recurrence_v1_reduce_resolved",
                     "pacman_recurrence_v1_reduce_sample", "pacman_recurrence_v1_configure"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_int
        L.pacman_recurrence_v1_capabilities.restype = C.c_uint32
        L.pacman_recurrence_v1_symjit_kernel.argtypes = [C.c_char_p]
        L.pacman_recurrence_v1_host_alloc.argtypes = [C.c_size_t]
        L.pacman_recurrence_v1_host_alloc.restype = C.c_void_p
        L.pacman_recurrence_v1_host_free.argtypes = [C.c_void_p]
        L.pacman_recurrence_v1_test_sources.argtypes = [C.c_void_p] * 3 + [C.c_uint32] + [C.c_void_p] * 2
        if kernel is not None:
            self.configure(kernel, block, no_sort, stats, executor)

    def configure(self, kernel="f64", block=0, no_sort=False, stats=False, executor=None, lanes_per_point=0):
        o = abi.options(kernel, block, no_sort, stats, executor, lanes_per_point)
        return self.lib.pacman_recurrence_v1_configure(C.addressof(o))

    def run(self, call_args):
        return self.lib.pacman_recurrence_v1_run(C.addressof(call_args.struct))

    def reduce_resolved(self, r):
        return self.lib.pacman_recurrence_v1_reduce_resolved(C.addressof(r))

    def reduce(self, r):
        return self.lib.pacman_recurrence_v1_reduce(C.addressof(r))

    def reduce_sample(self, r):
        return self.lib.pacman_recurrence_v1_reduce_sample(C.addressof(r))

    def capabilities(self):
        return self.lib.pacman_recurrence_v1_capabilities()

    def symjit_kernel(self, sha):
        return self.lib.pacman_recurrence_v1_symjit_kernel(sha if sha is None else sha.encode())

    def test_sources(self, codes, masses, momenta):
        codes = np.ascontiguousarray(codes, dtype=np.uint32)
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        momenta = np.ascontiguousarray(momenta, dtype=np.float64)
        n = len(codes)
        re, im = np.zeros(4 * n), np.zeros(4 * n)
        status = self.lib.pacman_recurrence_v1_test_sources(codes.ctypes.data, masses.ctypes.data, momenta.ctypes.data,
                                                            n, re.ctypes.data, im.ctypes.data)
        if status != 0:
            raise RunnerError(f"test_sources returned {status}")
        return re.reshape(n, 4) + 1j * im.reshape(n, 4)

    def evaluate(self, template, momenta, resolved=True):
        """Amplitudes and resolved outputs of `template` at point-major momenta, as
        oracle.evaluate computes them: one run keeping its amplitudes... here the amplitudes
        are downloaded, then a second kept run is reduced on the device."""
        from . import phase_space

        points = momenta.shape[0]
        ext = phase_space.source_major(momenta)
        args = template.call(ext, points, flags=abi.FORMS_ON_DEVICE)
        status = self.run(args)
        if status != 0:
            raise RunnerError(f"run returned {status}")
        amps = (args.are + 1j * args.aim).reshape(template.amplitude_planes, points)
        out = None
        if resolved:
            keep = template.call(ext, points)
            status = self.run(keep)
            if status != 0:
                raise RunnerError(f"kept run returned {status}")
            out = np.zeros(points * template.outputs)
            r, hold = abi.reduce_resolved_args(template.planes, template.weights, template.offsets, out, points, 1,
                                               template.outputs, abi.OUTPUT_ZERO)
            status = self.reduce_resolved(r)
            if status != 0:
                raise RunnerError(f"reduce_resolved returned {status}")
            out = out.reshape(points, template.outputs)
        return amps, out
