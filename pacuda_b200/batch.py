"""The batched, device-resident API (include/pacuda_b200.h) from Python, with torch tensors as
device memory."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .runner import DEFAULT_LIB, RunnerError

_lib = None


def lib(path=None):
    global _lib
    if _lib is None:
        _lib = C.CDLL(path or DEFAULT_LIB)
        L = _lib
        L.pacuda_b200_plan_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]
        L.pacuda_b200_plan_create.restype = C.c_void_p
        L.pacuda_b200_plan_destroy.argtypes = [C.c_void_p]
        L.pacuda_b200_plan_flops.argtypes = [C.c_void_p]
        L.pacuda_b200_plan_flops.restype = C.c_uint64
        L.pacuda_b200_plan_set_lanes_per_point.argtypes = [C.c_void_p, C.c_uint32]
        L.pacuda_b200_plan_lanes_per_point.argtypes = [C.c_void_p]
        L.pacuda_b200_plan_lanes_per_point.restype = C.c_uint32
        L.pacuda_b200_batch_create.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.pacuda_b200_batch_create.restype = C.c_void_p
        for name in ("pacuda_b200_batch_tune", "pacuda_b200_batch_run", "pacuda_b200_batch_capture"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_void_p]
        L.pacuda_b200_batch_launches.argtypes = [C.c_void_p]
        L.pacuda_b200_batch_launches.restype = C.c_uint32
        L.pacuda_b200_batch_set_blocks_per_sm.argtypes = [C.c_void_p, C.c_uint32]
        L.pacuda_b200_batch_blocks_per_sm.argtypes = [C.c_void_p]
        L.pacuda_b200_batch_blocks_per_sm.restype = C.c_uint32
        L.pacuda_b200_batch_lanes_per_point.argtypes = [C.c_void_p, C.c_uint32]
        L.pacuda_b200_batch_lanes_per_point.restype = C.c_uint32
        L.pacuda_b200_batch_plan_blocks_per_sm.argtypes = [C.c_void_p, C.c_uint32]
        L.pacuda_b200_batch_set_plan_blocks_per_sm.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.pacuda_b200_batch_plan_blocks_per_sm.restype = C.c_uint32
        L.pacuda_b200_batch_update.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.pacuda_b200_batch_destroy.argtypes = [C.c_void_p]
    return _lib


class Plan:
    """A compiled plan (a `plan.Template`) for the batched executor."""

    def __init__(self, template, kernel="f64"):
        self.template = template
        k = abi.BATCH_KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        args = template.call(np.zeros(4 * template.external_count), 1)
        self._keep = (np.ascontiguousarray(template.offsets, dtype=np.uint32),
                      np.ascontiguousarray(template.planes, dtype=np.uint32),
                      np.ascontiguousarray(template.weights, dtype=np.float64), args)
        off, planes, weights, _ = self._keep
        self.handle = lib().pacuda_b200_plan_create(C.addressof(args.struct), off.ctypes.data, planes.ctypes.data,
                                                    weights.ctypes.data, template.outputs, k)
        if not self.handle:
            raise RunnerError("pacuda_b200_plan_create failed")

    @property
    def flops(self):
        return lib().pacuda_b200_plan_flops(self.handle)

    @property
    def lanes_per_point(self):
        return lib().pacuda_b200_plan_lanes_per_point(self.handle)

    @lanes_per_point.setter
    def lanes_per_point(self, n):
        if lib().pacuda_b200_plan_set_lanes_per_point(self.handle, n) != 0:
            raise RunnerError(f"{n} lanes per point do not fit")

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.pacuda_b200_plan_destroy(self.handle)
            self.handle = None


class Batch:
    """Plans evaluated together: plan k on the device momenta `external[k]` (a float64 CUDA
    tensor of source-major planes) into `output[k]` (float64 CUDA tensor [points][outputs])."""

    def __init__(self, plans, external, output):
        import torch

        self.plans, self.external, self.output = list(plans), list(external), list(output)
        n = len(self.plans)
        self.counts = [int(e.numel() // (4 * p.template.external_count)) for p, e in zip(self.plans, self.external)]
        for p, o, c in zip(self.plans, self.output, self.counts):
            assert o.dtype == torch.float64 and o.is_cuda and o.numel() == c * p.template.outputs
        handles = (C.c_void_p * n)(*[p.handle for p in self.plans])
        ext = (C.c_void_p * n)(*[e.data_ptr() for e in self.external])
        out = (C.c_void_p * n)(*[o.data_ptr() for o in self.output])
        cnt = (C.c_uint32 * n)(*self.counts)
        self.handle = lib().pacuda_b200_batch_create(handles, n, ext, cnt, out)
        if not self.handle:
            raise RunnerError("pacuda_b200_batch_create failed")

    def update(self, external, counts, output):
        """Points the plans at other momenta, point counts and outputs (pacuda_b200_batch_update:
        no allocation; a captured graph is dropped)."""
        import torch

        n = len(self.plans)
        external, output, counts = list(external), list(output), [int(c) for c in counts]
        assert len(external) == len(output) == len(counts) == n
        for p, e, o, c in zip(self.plans, external, output, counts):
            assert e.dtype == torch.float64 and e.is_cuda and e.numel() >= 4 * p.template.external_count * c
            assert o.dtype == torch.float64 and o.is_cuda and o.numel() >= c * p.template.outputs
        ext = (C.c_void_p * n)(*[e.data_ptr() for e in external])
        out = (C.c_void_p * n)(*[o.data_ptr() for o in output])
        cnt = (C.c_uint32 * n)(*counts)
        if lib().pacuda_b200_batch_update(self.handle, ext, cnt, out) != 0:
            raise RunnerError("batch update failed")
        self.external, self.output, self.counts = external, output, counts

    def _stream(self, stream):
        import torch

        s = stream if stream is not None else torch.cuda.current_stream()
        return C.c_void_p(s.cuda_stream)

    def tune(self, stream=None):
        if lib().pacuda_b200_batch_tune(self.handle, self._stream(stream)) != 0:
            raise RunnerError("tune failed")

    def run(self, stream=None):
        if lib().pacuda_b200_batch_run(self.handle, self._stream(stream)) != 0:
            raise RunnerError("batch run failed")

    def capture(self, stream=None):
        if lib().pacuda_b200_batch_capture(self.handle, self._stream(stream)) != 0:
            raise RunnerError("capture failed")

    @property
    def launches(self):
        return lib().pacuda_b200_batch_launches(self.handle)

    def lanes_per_point(self, k):
        """The lanes per point plan k runs with in this batch's launch."""
        return lib().pacuda_b200_batch_lanes_per_point(self.handle, k)

    def plan_blocks_per_sm(self, k):
        """The blocks per SM plan k runs with."""
        return lib().pacuda_b200_batch_plan_blocks_per_sm(self.handle, k)

    def set_plan_blocks_per_sm(self, k, blocks):
        if lib().pacuda_b200_batch_set_plan_blocks_per_sm(self.handle, k, blocks) != 0:
            raise RunnerError(f"plan {k}: {blocks} blocks per SM do not fit")

    @property
    def blocks_per_sm(self):
        return lib().pacuda_b200_batch_blocks_per_sm(self.handle)

    @blocks_per_sm.setter
    def blocks_per_sm(self, n):
        if lib().pacuda_b200_batch_set_blocks_per_sm(self.handle, n) != 0:
            raise RunnerError(f"{n} blocks per SM do not fit")

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.pacuda_b200_batch_destroy(self.handle)
            self.handle = None
