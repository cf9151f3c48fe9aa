"""Mixed precision with a rotated-momentum stability check, on the batched executor.

Each point's |M|^2 is evaluated by the mixed kernel (f32 currents, df64 denominators and
amplitudes) twice: at its momenta and at the same momenta turned by one fixed spatial rotation.
|M|^2 is rotation invariant, so the two totals differ only by the kernel's rounding; a point whose
totals differ by more than `tol` (relative), or are not finite, is evaluated again by the f64
kernel, and its f64 outputs replace its mixed ones. The f64 kernel is the reference runner's f64
arithmetic, so a point sent back carries the f64 bits.

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


def rotate(ext, legs, rot):
    """Source-major momenta `ext` ([(leg * 4 + k) * n + i], a float64 tensor) with every leg's
    spatial components turned by `rot` (3x3); energies unchanged. A new tensor."""
    import torch

    n = ext.numel() // (4 * legs)
    e = ext.view(legs, 4, n)
    r = torch.as_tensor(rot, dtype=torch.float64, device=ext.device)
    out = torch.empty_like(e)
    out[:, 0, :] = e[:, 0, :]
    out[:, 1:, :] = torch.einsum("ij,ljn->lin", r, e[:, 1:, :])
    return out.view(-1)


class StableMixed:
    """Plans of one process (a list of `plan.Template`, whose outputs add up: a process's plan
    parts, or one template) over `points` points: mixed outputs, with the points that fail the
    rotation check evaluated again in f64."""

    def __init__(self, templates, points, tol, seed=7):
        import torch

        self.templates = list(templates)
        self.points = int(points)
        self.tol = float(tol)
        self.legs = self.templates[0].external_count
        self.rot = rotation(seed)
        self.mixed = [B.Plan(t, "mixed") for t in self.templates]
        self.f64 = [B.Plan(t, "f64") for t in self.templates]
        dev = "cuda"
        self.out = [torch.empty(self.points * t.outputs, dtype=torch.float64, device=dev) for t in self.templates]
        self.out_rot = [torch.empty_like(o) for o in self.out]
        self._mixed_batch = self._f64_batch = None
        self._ext = self._ext_rot = None
        self.unstable = None  # the last run's mask of points sent to f64 (bool tensor)

    def _totals(self, outs):
        n = self.points
        return sum(o.view(n, t.outputs).sum(dim=1) for o, t in zip(outs, self.templates))

    def run(self, ext):
        """Evaluates the points of `ext` (source-major float64 CUDA tensor for `points` points);
        returns the per-template outputs ([points][outputs] each) and the number of points that
        went back to f64."""
        import torch

        n, P = self.points, len(self.templates)
        assert ext.numel() == 4 * self.legs * n and ext.dtype == torch.float64 and ext.is_cuda
        self._ext = ext
        self._ext_rot = rotate(ext, self.legs, self.rot)
        exts = [self._ext] * P + [self._ext_rot] * P
        outs = self.out + self.out_rot
        if self._mixed_batch is None:
            self._mixed_batch = B.Batch(self.mixed + self.mixed, exts, outs)
        else:
            self._mixed_batch.update(exts, [n] * (2 * P), outs)
        self._mixed_batch.run()
        a, b = self._totals(self.out), self._totals(self.out_rot)
        rel = (a - b).abs() / a.abs().clamp_min(1e-300)
        self.unstable = ~(rel <= self.tol)
        idx = torch.nonzero(self.unstable).flatten()
        m = int(idx.numel())
        if m:
            sel = self._ext.view(4 * self.legs, n).index_select(1, idx).contiguous().view(-1)
            sel_out = [torch.empty(m * t.outputs, dtype=torch.float64, device=ext.device) for t in self.templates]
            if self._f64_batch is None:
                self._f64_batch = B.Batch(self.f64, [sel] * P, sel_out)
            else:
                self._f64_batch.update([sel] * P, [m] * P, sel_out)
            self._f64_batch.run()
            for o, s, t in zip(self.out, sel_out, self.templates):
                o.view(n, t.outputs)[idx] = s.view(m, t.outputs)
        return self.out, m
