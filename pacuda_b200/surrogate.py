"""The surrogate network (include/pacuda_surrogate.h, libsurrogate.so) from Python, with torch
tensors as device memory. The product path has no fallback: a missing library is an error."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsurrogate.so")
WIDTH = 256
MAX_INPUTS = 64
_lib = None


class SurrogateError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise SurrogateError(f"{LIB}: not built (python -m pacuda_b200.build)")
        L = C.CDLL(LIB)
        L.pacuda_sg_param_count.restype = C.c_size_t
        L.pacuda_sg_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        L.pacuda_sg_create.restype = C.c_void_p
        L.pacuda_sg_destroy.argtypes = [C.c_void_p]
        L.pacuda_sg_set_params.argtypes = [C.c_void_p, C.c_void_p]
        L.pacuda_sg_get_params.argtypes = [C.c_void_p, C.c_void_p]
        L.pacuda_sg_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
        L.pacuda_sg_train_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p,
                                           C.c_void_p]
        L.pacuda_sg_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.pacuda_sg_last_launches.restype = C.c_uint32
        L.pacuda_sg_error.argtypes = [C.c_void_p]
        L.pacuda_sg_set_inference_blocks.argtypes = [C.c_uint32]
        L.pacuda_sg_apply_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]
        _lib = L
    return _lib


def param_count():
    return int(lib().pacuda_sg_param_count())


def _stream(stream):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _check(status, what):
    if status != 0:
        raise SurrogateError(f"{what} returned {status}")


class Network:
    """A network of `inputs` features with training workspace for batches of `max_batch` points."""

    def __init__(self, inputs, max_batch=16384, seed=1):
        self.inputs, self.max_batch = int(inputs), int(max_batch)
        self.handle = lib().pacuda_sg_create(self.inputs, self.max_batch, seed)
        if not self.handle:
            raise SurrogateError("pacuda_sg_create failed")

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.pacuda_sg_destroy(self.handle)
            self.handle = None

    def params(self):
        p = np.zeros(param_count(), dtype=np.float32)
        _check(lib().pacuda_sg_get_params(self.handle, p.ctypes.data), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == param_count()
        _check(lib().pacuda_sg_set_params(self.handle, p.ctypes.data), "set_params")

    def gradients(self, x, y, stream=None):
        import torch

        grad = torch.empty(param_count(), dtype=torch.float32, device=x.device)
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        _check(lib().pacuda_sg_gradients(self.handle, x.data_ptr(), y.data_ptr(), x.shape[0], grad.data_ptr(),
                                         loss.data_ptr(), _stream(stream)), "gradients")
        return grad, loss

    def train_step(self, x, y, lr, loss_sum=None, stream=None):
        _check(lib().pacuda_sg_train_step(self.handle, x.data_ptr(), y.data_ptr(), x.shape[0], float(lr),
                                          loss_sum.data_ptr() if loss_sum is not None else None, _stream(stream)),
               "train_step")

    def apply_gradients(self, grad, lr, stream=None):
        """One Adam step on a supplied gradient (a float32 CUDA tensor in parameter order)."""
        _check(lib().pacuda_sg_apply_gradients(self.handle, grad.data_ptr(), float(lr), _stream(stream)),
               "apply_gradients")

    def forward(self, x, out=None, stream=None):
        import torch

        n = x.shape[0]
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=x.device)
        _check(lib().pacuda_sg_forward(self.handle, x.data_ptr(), n, out.data_ptr(), _stream(stream)), "forward")
        return out

    def error(self):
        return lib().pacuda_sg_error(self.handle)


def set_inference_blocks(blocks):
    """Blocks per SM of the fused inference kernel (1 or 2)."""
    _check(lib().pacuda_sg_set_inference_blocks(int(blocks)), "set_inference_blocks")


def last_launches():
    return int(lib().pacuda_sg_last_launches())
