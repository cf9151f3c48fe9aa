"""ctypes mirror of the recurrence runner's C ABI (include/pacman_recurrence.h).

The structs are the reference's binary layout (runner/pacman_recurrence.h:18-145); this module
only builds them from numpy arrays and keeps the arrays alive for the duration of a call.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

ABI = 1
KEEP_AMPLITUDES = 1
FORMS_ON_DEVICE = 2
OUTPUT_ZERO = 1
OK, INVALID, DEVICE_ERROR = 0, 2, 3
KERNEL_DF64, KERNEL_F64, KERNEL_MIXED, KERNEL_MIXED64 = 0, 1, 2, 3
KERNELS = {"df64": KERNEL_DF64, "f64": KERNEL_F64, "mixed": KERNEL_MIXED, "mixed64": KERNEL_MIXED64}
KERNEL_F64_FMA = 4  # the batched API's f64 kind with contracted multiply-adds (include/pacuda_b200.h)
BATCH_KERNELS = dict(KERNELS, f64fma=KERNEL_F64_FMA)
CAP_SOURCES, CAP_FORMS, CAP_SYMJIT = 1, 2, 4
W_P, W_A, W_F, W_X, W_S, W_K = range(6)

_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_U64 = C.POINTER(C.c_uint64)


class Call(C.Structure):
    """pacman_recurrence_call (reference: runner/pacman_recurrence.h:18-51)."""

    _fields_ = [
        ("abi_version", C.c_uint32), ("struct_size", C.c_uint32),
        ("words", _U64), ("words_key", C.c_uint64), ("word_count", C.c_uint32),
        ("width", C.c_uint8 * 8),
        ("current_re", _D), ("current_im", _D), ("amplitude_re", _D), ("amplitude_im", _D),
        ("momenta", _D), ("scale_re", _D), ("scale_im", _D), ("factor_re", _D), ("factor_im", _D),
        ("upload_current", _U32), ("upload_amplitude", _U32), ("download_amplitude", _U32),
        ("download_current", _U32),
        ("current_planes", C.c_uint32), ("amplitude_planes", C.c_uint32), ("momentum_planes", C.c_uint32),
        ("scale_count", C.c_uint32), ("factor_count", C.c_uint32),
        ("upload_current_runs", C.c_uint32), ("upload_amplitude_runs", C.c_uint32),
        ("download_amplitude_runs", C.c_uint32), ("download_current_runs", C.c_uint32),
        ("stride", C.c_uint32), ("points", C.c_uint32),
        ("zero_amplitude", _U32), ("zero_amplitude_runs", C.c_uint32), ("flags", C.c_uint32),
        ("external_momenta", _D), ("external_count", C.c_uint32), ("term_count", C.c_uint32),
        ("form_terms", _U32), ("term_slots", _U32), ("term_coefficients", _D),
    ]


CALL_V1_SIZE = Call.zero_amplitude.offset
CALL_V2_SIZE = Call.external_momenta.offset


class Reduce(C.Structure):
    """pacman_recurrence_reduce (reference: runner/pacman_recurrence.h:62-69)."""

    _fields_ = [("abi_version", C.c_uint32), ("struct_size", C.c_uint32), ("planes", _U32),
                ("weights", _D), ("output", _D), ("count", C.c_uint32), ("points", C.c_uint32)]


class ReduceResolved(C.Structure):
    """pacman_recurrence_reduce_resolved (reference: runner/pacman_recurrence.h:85-94)."""

    _fields_ = [("abi_version", C.c_uint32), ("struct_size", C.c_uint32), ("planes", _U32),
                ("weights", _D), ("offsets", _U32), ("output", _D), ("outputs", C.c_uint32),
                ("points", C.c_uint32), ("output_stride", C.c_uint32), ("point_stride", C.c_uint32),
                ("flags", C.c_uint32)]


class ReduceSample(C.Structure):
    """pacman_recurrence_reduce_sample (reference: runner/pacman_recurrence.h:105-118)."""

    _fields_ = [("abi_version", C.c_uint32), ("struct_size", C.c_uint32), ("planes", _U32),
                ("weights", _D), ("offsets", _U32), ("helicity", _U32), ("outputs", C.c_uint32),
                ("points", C.c_uint32), ("random", _D), ("scale", _D), ("numerator", C.c_double),
                ("denominator", C.c_double), ("total", _D), ("chosen", _U32)]


class Options(C.Structure):
    """pacman_recurrence_options (reference: runner/pacman_recurrence.h:131-138)."""

    _fields_ = [("abi_version", C.c_uint32), ("struct_size", C.c_uint32), ("kernel", C.c_uint32),
                ("block", C.c_uint32), ("no_sort", C.c_uint32), ("stats", C.c_uint32)]


def ptr(a, kind):
    """A ctypes pointer to numpy array `a` (or NULL for None)."""
    if a is None:
        return C.cast(None, kind)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays passed to the runner must be C-contiguous")
    return a.ctypes.data_as(kind)


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def u32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint32)


def runs_of(a):
    """(array, run count) of a flat (first, count) list."""
    a = u32(a)
    return (a, 0) if a is None else (a, len(a) // 2)


class CallArgs:
    """A `Call` built from numpy arrays; holds the arrays so their memory outlives the call.

    `current` / `amplitude` are (re, im) pairs of float64 arrays of planes * stride values.
    """

    def __init__(self, *, words, width, stride, points, current, amplitude, current_planes,
                 amplitude_planes, momentum_planes=0, momenta=None, scales=((), ()),
                 factors=((), ()), upload_current=None, upload_amplitude=None,
                 download_amplitude=None, download_current=None, zero_amplitude=None, flags=0,
                 external=None, external_count=0, form_terms=None, term_slots=None,
                 term_coefficients=None, words_key=0, struct_size=None):
        self.words = np.ascontiguousarray(words, dtype=np.uint64)
        self.cre, self.cim = current
        self.are, self.aim = amplitude
        self.momenta = f64(momenta)
        self.sre, self.sim = f64(np.asarray(scales[0], dtype=np.float64)), f64(np.asarray(scales[1], dtype=np.float64))
        self.fre, self.fim = f64(np.asarray(factors[0], dtype=np.float64)), f64(np.asarray(factors[1], dtype=np.float64))
        self.up_c, n_up_c = runs_of(upload_current)
        self.up_a, n_up_a = runs_of(upload_amplitude)
        self.down_a, n_down_a = runs_of(download_amplitude)
        self.down_c, n_down_c = runs_of(download_current)
        self.zero, n_zero = runs_of(zero_amplitude)
        self.external = f64(external)
        self.form_terms = u32(form_terms)
        self.term_slots = u32(term_slots)
        self.term_coefficients = f64(term_coefficients)
        c = Call()
        c.abi_version = ABI
        c.struct_size = C.sizeof(Call) if struct_size is None else struct_size
        c.words = ptr(self.words, _U64)
        c.words_key = words_key
        c.word_count = len(self.words)
        for k in range(8):
            c.width[k] = int(width[k]) if k < len(width) else 0
        c.current_re, c.current_im = ptr(self.cre, _D), ptr(self.cim, _D)
        c.amplitude_re, c.amplitude_im = ptr(self.are, _D), ptr(self.aim, _D)
        c.momenta = ptr(self.momenta, _D)
        c.scale_re, c.scale_im = ptr(self.sre, _D), ptr(self.sim, _D)
        c.factor_re, c.factor_im = ptr(self.fre, _D), ptr(self.fim, _D)
        c.upload_current, c.upload_amplitude = ptr(self.up_c, _U32), ptr(self.up_a, _U32)
        c.download_amplitude, c.download_current = ptr(self.down_a, _U32), ptr(self.down_c, _U32)
        c.current_planes, c.amplitude_planes, c.momentum_planes = current_planes, amplitude_planes, momentum_planes
        c.scale_count, c.factor_count = len(self.sre), len(self.fre)
        c.upload_current_runs, c.upload_amplitude_runs = n_up_c, n_up_a
        c.download_amplitude_runs, c.download_current_runs = n_down_a, n_down_c
        c.stride, c.points = stride, points
        c.zero_amplitude, c.zero_amplitude_runs = ptr(self.zero, _U32), n_zero
        c.flags = flags
        c.external_momenta = ptr(self.external, _D)
        c.external_count = external_count
        c.term_count = 0 if self.term_slots is None else len(self.term_slots)
        c.form_terms, c.term_slots = ptr(self.form_terms, _U32), ptr(self.term_slots, _U32)
        c.term_coefficients = ptr(self.term_coefficients, _D)
        self.struct = c

    def byref(self):
        return C.byref(self.struct)


def reduce_resolved_args(planes, weights, offsets, output, points, output_stride, point_stride, flags=0):
    planes, weights, offsets = u32(planes), f64(weights), u32(offsets)
    r = ReduceResolved(ABI, C.sizeof(ReduceResolved), ptr(planes, _U32), ptr(weights, _D), ptr(offsets, _U32),
                       ptr(output, _D), len(offsets) - 1, points, output_stride, point_stride, flags)
    return r, (planes, weights, offsets, output)


def reduce_args(planes, weights, output, points):
    planes, weights = u32(planes), f64(weights)
    r = Reduce(ABI, C.sizeof(Reduce), ptr(planes, _U32), ptr(weights, _D), ptr(output, _D), len(planes), points)
    return r, (planes, weights, output)


def reduce_sample_args(planes, weights, offsets, helicity, points, random, scale, numerator, denominator,
                       total, chosen):
    planes, weights, offsets, helicity = u32(planes), f64(weights), u32(offsets), u32(helicity)
    random, scale = f64(random), f64(scale)
    r = ReduceSample(ABI, C.sizeof(ReduceSample), ptr(planes, _U32), ptr(weights, _D), ptr(offsets, _U32),
                     ptr(helicity, _U32), len(offsets) - 1, points, ptr(random, _D), ptr(scale, _D),
                     numerator, denominator, ptr(total, _D), ptr(chosen, _U32))
    return r, (planes, weights, offsets, helicity, random, scale, total, chosen)


class B200Options(C.Structure):
    """pacuda_b200_options (include/pacuda_b200.h): the reference's options, then the executor and
    the on-chip executor's lanes per point."""

    _fields_ = [("base", Options), ("executor", C.c_uint32), ("lanes_per_point", C.c_uint32)]


EXECUTORS = {"auto": 0, "arena": 1, "onchip": 2}


def options(kernel="f64", block=0, no_sort=False, stats=False, executor=None, lanes_per_point=0):
    """The configuration struct: the reference's, or this library's larger one when an executor
    or lanes per point is given."""
    k = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
    base = Options(ABI, C.sizeof(Options), k, block, 1 if no_sort else 0, 1 if stats else 0)
    if executor is None and not lanes_per_point:
        return base
    base.struct_size = C.sizeof(B200Options)
    return B200Options(base, EXECUTORS[executor or "auto"], lanes_per_point)
