"""Recurrence plans: rows, their 64-bit words, and a run template.

A plan is a list of rows that the runner executes per phase-space point. Each row is one 64-bit
word: the op in the low 4 bits, then the op's fields, each as wide as the plan's `width` table
says (reference: runner/recurrence_runner.cu:10-36 describes the layout; convert/src/program.rs
:60-162 decodes and encodes it). This module is the Python side of that format: `encode` and
`decode` are inverses, and `Template` holds one run's static tables (as a `.pacuda` colour's
template, convert/src/format.rs:19-26) plus the reduction into helicity outputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import abi

W_P, W_A, W_F, W_X, W_S, W_K = range(6)

# (op, field kinds) of every one-word op, fields in word order (program.rs:90-107)
_LAYOUT = {
    1: ("P", "P"),
    2: ("1", "S", "P", "P", "P", "F", "F", "X"),
    7: ("P", "F", "X"),
    10: ("P", "K", "X"),
    11: ("P", "P", "A", "X", "X", "K"),
    12: ("P", "F", "X", "S", "10"),
    13: ("1", "P", "P", "P", "F", "F", "X"),
}
for _op in (3, 4, 5, 6):
    _LAYOUT[_op] = _LAYOUT[2]
for _op in (8, 9):
    _LAYOUT[_op] = _LAYOUT[7]
_INDEX = {"P": W_P, "A": W_A, "F": W_F, "X": W_X, "S": W_S, "K": W_K}


def contribution_shape(op):
    """(components of parent 0, of parent 1, written) of contribution op 2..6."""
    c0 = 6 if op == 4 else 4 if op in (5, 6) else 2
    cd = 4 if op in (4, 6) else 6 if op == 5 else 2
    return c0, 4, cd


def _bits(kind, width):
    if kind == "1":
        return 1
    if kind == "10":
        return 10
    return int(width[_INDEX[kind]])


def encode(rows, width):
    """The words of `rows`: each row a tuple (op, field, field, ...) in word order."""
    words = []
    for n, row in enumerate(rows):
        op, values = row[0], row[1:]
        layout = _LAYOUT.get(op)
        if layout is None or len(values) != len(layout):
            raise ValueError(f"row {n}: op {op} with {len(values)} fields")
        word, at = op, 4
        for value, kind in zip(values, layout):
            bits = _bits(kind, width)
            value = int(value)
            if value < 0 or (bits < 64 and value >> bits):
                raise ValueError(f"row {n}: {value} does not fit {bits} bits")
            word |= value << at
            at += bits
        if at > 64:
            raise ValueError(f"row {n}: {at} bits")
        words.append(word)
    return np.array(words, dtype=np.uint64)


def decode(words, width):
    """The rows of `words` (inverse of `encode`; op 14 rows are (14, kernel, n_in, pairs,
    direct, codes))."""
    rows, n = [], 0
    words = [int(w) for w in words]
    while n < len(words):
        w = words[n]
        if w & 15 == 14:
            kernel, n_in, pairs, direct = (w >> 4) & 0xFFFF, (w >> 20) & 0xFF, (w >> 28) & 0xFF, (w >> 36) & 1
            codes = []
            for k in range(n_in + pairs):
                d = words[n + 1 + k // 2] if n + 1 + k // 2 < len(words) else 0
                codes.append((d >> 32) if k % 2 else d & 0xFFFFFFFF)
            rows.append((14, kernel, n_in, pairs, direct, tuple(codes)))
            n += 1 + (n_in + pairs + 1) // 2
            continue
        op = w & 15
        layout = _LAYOUT.get(op)
        if layout is None:
            raise ValueError(f"word {n}: op {op}")
        w >>= 4
        values = []
        for kind in layout:
            bits = _bits(kind, width)
            values.append(w & ((1 << bits) - 1))
            w >>= bits
        rows.append((op, *values))
        n += 1
    return rows


def bits_for(n):
    """The width of a field holding values 0 .. n (at least 1 bit)."""
    return max(1, int(n).bit_length())


def widths_for(rows, current_planes, amplitude_planes, forms, factors, slots, k_max=None):
    """The narrowest width table for these rows (as RustiCol sizes them: the largest index of each
    kind; K from the largest count)."""
    k = k_max if k_max is not None else max(
        [r[2] for r in rows if r[0] == 10] + [r[6] for r in rows if r[0] == 11] + [1])
    width = [bits_for(current_planes), bits_for(max(0, amplitude_planes - 1)), bits_for(max(0, forms - 1)),
             bits_for(max(0, factors - 1)), bits_for(max(0, slots - 1)), bits_for(k), 0, 0]
    return width


def source_code(family, orientation, helicity, chirality):
    """The 10-bit template code of an op 12 row (recurrence_runner.cu:25-28, :529-531)."""
    return family | orientation << 3 | (helicity + 2) << 5 | (chirality + 1) << 8


@dataclass
class Template:
    """One run's static part and its reduction (a `.pacuda` colour, convert/src/format.rs:19-28).

    Forms are built on the device from `external_count` external momenta: form f is
    sum_t coefficient_t * p(slot_t) over its terms `form_terms[2f] ..` (first, count)."""

    words: np.ndarray
    width: list
    current_planes: int
    amplitude_planes: int
    momentum_planes: int
    scale_re: np.ndarray
    scale_im: np.ndarray
    factor_re: np.ndarray
    factor_im: np.ndarray
    zero_amplitude: np.ndarray          # runs (first, count) flattened
    download_amplitude: np.ndarray      # runs
    external_count: int
    form_terms: np.ndarray              # (first, count) per form, flattened
    term_slots: np.ndarray
    term_coefficients: np.ndarray
    offsets: np.ndarray                 # reduction: outputs + 1
    planes: np.ndarray
    weights: np.ndarray
    tile: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def outputs(self):
        return len(self.offsets) - 1

    def key(self):
        """The runner's program cache key: FNV-1a of the widths and the words (as UMAMI keys a
        program, umami/umami_pacuda.c:300-307), never 0."""
        h = 1469598103934665603
        data = bytes(bytearray(int(b) & 0xFF for b in self.width[:8])) + np.asarray(self.words, dtype="<u8").tobytes()
        for b in data:
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return h or 1

    def call(self, external, points, stride=None, flags=abi.KEEP_AMPLITUDES | abi.FORMS_ON_DEVICE,
             current=None, amplitude=None, words_key=None):
        """The CallArgs of one tile: `external` source-major planes [(l * 4 + k) * points + i]."""
        stride = stride or points
        if current is None:
            current = (np.zeros(self.current_planes * stride), np.zeros(self.current_planes * stride))
        if amplitude is None:
            amplitude = (np.zeros(self.amplitude_planes * stride), np.zeros(self.amplitude_planes * stride))
        return abi.CallArgs(
            words=self.words, width=self.width, stride=stride, points=points, current=current,
            amplitude=amplitude, current_planes=self.current_planes, amplitude_planes=self.amplitude_planes,
            momentum_planes=self.momentum_planes, momenta=np.zeros(max(1, self.momentum_planes * stride)),
            scales=(self.scale_re, self.scale_im), factors=(self.factor_re, self.factor_im),
            download_amplitude=self.download_amplitude, zero_amplitude=self.zero_amplitude, flags=flags,
            external=external, external_count=self.external_count, form_terms=self.form_terms,
            term_slots=self.term_slots, term_coefficients=self.term_coefficients,
            words_key=self.key() if words_key is None else words_key)
