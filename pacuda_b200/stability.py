"""Mixed precision with a rotated-momentum stability check, on the batched executor.

Each point's |M|^2 is evaluated by the mixed kernel (f32 currents, df64 denominators and
amplitudes) twice: at its momenta and at the same momenta turned by one fixed spatial rotation.
|M|^2 is rotation invariant, so the two totals differ only by the kernel's rounding; a point whose
totals differ by more than `tol` (relative), or are not finite, is evaluated again by the f64
kernel, and its f64 outputs replace its mixed ones. The f64 kernel is the reference runner's f64
arithmetic, so a point sent back carries the f64 bits.

The check estimates a point's error; it does not bound it: both evaluations round their f32
currents alike, so a kept point's error can exceed `tol` (a few times tol on g g -> 4 g at
tol = 1e-6). Below FLOOR the check is not used at all.

The reference's runner has no such check (its mixed kinds are `recurrence_runner.cu:181-218`);
this is the fallback of the precision pattern, measured by the gg -> 4g line of the benchmark.
"""
from __future__ import annotations

import numpy as np

from . import batch as B


def rotation(seed):
    """A fixed 3x3 rotation (f64): seeded axis and angle, by Rodrigues' formula."""
    rng = np.random.default_rng(seed)
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    angle = rng.uniform(0.5, 2.5)
    k = np.array([[0.0, -axis[2], axis[1]], [axis[2], 0.0, -axis[0]], [-axis[1], axis[0], 0.0]])
    return np.eye(3) + np.sin(angle) * k + (1.0 - np.cos(angle)) * (k @ k)


# Two f32 evaluations can agree closely by chance while both are about 1e-7 off (the mixed
# kernel's rounding of its currents): a tolerance below this floor certifies nothing, so every
# point then goes to f64 (the mixed evaluations are skipped).
FLOOR = 1e-6


def _lib():
    import ctypes as C

    L = B.lib()
    if not getattr(L, "_stability_bound", False):
        L.pacuda_b200_rotate.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.pacuda_b200_compare.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_double,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
        L.pacuda_b200_gather.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                         C.c_void_p, C.c_void_p]
        L.pacuda_b200_scatter.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_void_p]
        L._stability_bound = True
    return L


def _check(status, what):
    if status != 0:
        raise B.RunnerError(f"{what} returned {status}")


def _stream():
    import ctypes as C

    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def rotate(ext, legs, rot):
    """Source-major momenta `ext` ([(leg * 4 + k) * n + i], a float64 tensor) with every leg's
    spatial components turned by `rot` (3x3); energies unchanged. A new tensor (on the device the
    library's rotation kernel, on the host the same formula in numpy)."""
    import ctypes as C

    import torch

    n = ext.numel() // (4 * legs)
    r = np.ascontiguousarray(rot, dtype=np.float64)
    if not ext.is_cuda:
        e = ext.view(legs, 4, n).numpy()
        out = np.empty_like(e)
        out[:, 0, :] = e[:, 0, :]
        for a in range(3):
            out[:, 1 + a, :] = r[a, 0] * e[:, 1, :] + r[a, 1] * e[:, 2, :] + r[a, 2] * e[:, 3, :]
        return torch.from_numpy(out.reshape(-1))
    out = torch.empty_like(ext)
    _check(_lib().pacuda_b200_rotate(C.c_void_p(ext.data_ptr()), legs, n, r.ctypes.data, C.c_void_p(out.data_ptr()),
                                     _stream()), "rotate")
    return out


class StableMixed:
    """Plans of one process (a list of `plan.Template`, whose outputs add up: a process's plan
    parts, or one template) over `points` points: mixed outputs, with the points that fail the
    rotation check evaluated again in f64. A tolerance below FLOOR sends every point to f64.

    One run: the rotation (a kernel), both mixed evaluations (one persistent launch), the
    comparison (a kernel appending the failing points to a device list), one read of their
    count, their momenta gathered (a kernel), their f64 evaluation (one launch) and their outputs
    put in place (a kernel)."""

    def __init__(self, templates, points, tol, seed=7):
        import torch

        self.templates = list(templates)
        self.points = int(points)
        self.tol = float(tol)
        self.direct = self.tol < FLOOR
        self.legs = self.templates[0].external_count
        self.rot = rotation(seed)
        self.mixed = [B.Plan(t, "mixed") for t in self.templates]
        self.f64 = [B.Plan(t, "f64") for t in self.templates]
        dev = "cuda"
        n = self.points
        self.out = [torch.empty(n * t.outputs, dtype=torch.float64, device=dev) for t in self.templates]
        self.out_rot = [torch.empty_like(o) for o in self.out]
        self.sel_out = [torch.empty(n * t.outputs, dtype=torch.float64, device=dev) for t in self.templates]
        self.sel = torch.empty(4 * self.legs * n, dtype=torch.float64, device=dev)
        self.ext_rot = torch.empty(4 * self.legs * n, dtype=torch.float64, device=dev)
        self.index = torch.empty(n, dtype=torch.int32, device=dev)
        self.count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ptr_a = torch.tensor([o.data_ptr() for o in self.out], dtype=torch.int64, device=dev)
        self.ptr_b = torch.tensor([o.data_ptr() for o in self.out_rot], dtype=torch.int64, device=dev)
        self.n_out = torch.tensor([t.outputs for t in self.templates], dtype=torch.int32, device=dev)
        self._mixed_batch = self._f64_batch = None
        self.unstable = None  # the last run's mask of points sent to f64 (bool tensor)

    def run(self, ext):
        """Evaluates the points of `ext` (source-major float64 CUDA tensor for `points` points);
        returns the per-template outputs ([points][outputs] each) and the number of points that
        went back to f64."""
        import ctypes as C

        import torch

        n, P = self.points, len(self.templates)
        assert ext.numel() == 4 * self.legs * n and ext.dtype == torch.float64 and ext.is_cuda
        if self.direct:
            if self._f64_batch is None:
                self._f64_batch = B.Batch(self.f64, [ext] * P, self.out)
            else:
                self._f64_batch.update([ext] * P, [n] * P, self.out)
            self._f64_batch.run()
            self.unstable = torch.ones(n, dtype=torch.bool, device=ext.device)
            return self.out, n
        L = _lib()
        rot = np.ascontiguousarray(self.rot, dtype=np.float64)
        _check(L.pacuda_b200_rotate(C.c_void_p(ext.data_ptr()), self.legs, n, rot.ctypes.data,
                                    C.c_void_p(self.ext_rot.data_ptr()), _stream()), "rotate")
        exts = [ext] * P + [self.ext_rot] * P
        outs = self.out + self.out_rot
        if self._mixed_batch is None:
            self._mixed_batch = B.Batch(self.mixed + self.mixed, exts, outs)
        else:
            self._mixed_batch.update(exts, [n] * (2 * P), outs)
        self._mixed_batch.run()
        self.count.zero_()
        ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        _check(L.pacuda_b200_compare(ptr(self.ptr_a), ptr(self.ptr_b), ptr(self.n_out), P, n, self.tol,
                                     ptr(self.index), ptr(self.count), _stream()), "compare")
        m = int(self.count.item())
        self.unstable = torch.zeros(n, dtype=torch.bool, device=ext.device)
        if m:
            self.unstable[self.index[:m].long()] = True
            sel = self.sel[: 4 * self.legs * m]
            _check(L.pacuda_b200_gather(ptr(ext), self.legs, n, ptr(self.index), ptr(self.count), m, ptr(sel),
                                        _stream()), "gather")
            sel_out = [o[: m * t.outputs] for o, t in zip(self.sel_out, self.templates)]
            if self._f64_batch is None:
                self._f64_batch = B.Batch(self.f64, [sel] * P, sel_out)
            else:
                self._f64_batch.update([sel] * P, [m] * P, sel_out)
            self._f64_batch.run()
            for o, s, t in zip(self.out, sel_out, self.templates):
                _check(L.pacuda_b200_scatter(ptr(s), t.outputs, ptr(self.index), ptr(self.count), m, ptr(o),
                                             _stream()), "scatter")
        return self.out, m
