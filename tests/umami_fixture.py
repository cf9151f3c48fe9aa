"""A two-process UMAMI subprocess for the tests: the artifact (directory + `.pacuda` file), its
provider header, events, and every mode's expected |M|^2 from the oracle (test infrastructure).

Processes gg>ggg and qg>qgg (the latter with a crossing that swaps legs 3 and 4), channel 0 the
gluon process, channel 1 the quark one with three flavours: the identity, the two initial legs
swapped, and two contributions (factors 0.25 and 0.75, the second with legs 2 and 3 swapped).
The expected values follow the reference library's arithmetic (umami/umami_pacuda.c:700-749,
recurrence_runner.cu:1532-1572) in the same order, so the library must match them bit for bit.
"""
from __future__ import annotations

import math
import os

import numpy as np

from pacuda_b200 import pacuda_file, phase_space, processes

NAMES = ["gg>ggg", "qg>qgg"]
LEGS = 5
IDENTITY = [0, 1, 2, 3, 4]
SPEC = {
    "particles": LEGS, "masses": [0.0] * LEGS, "colors": 2,
    "processes": [{"key": "gg>ggg", "helicities": 32, "parameters": [("aS", 0.118, 0.0, False, True),
                                                                       ("MT", 173.0, 0.0, False, False)]},
                  {"key": "qg>qgg", "helicities": 32, "parameters": [("aS", 0.118, 0.0, False, True),
                                                                       ("ymt", 173.0, 0.0, False, True)]}],
    "channels": [
        [[{"process": 0, "colour": "lc", "permutation": IDENTITY, "factor": 1.0, "color_index": 0}]],
        [[{"process": 1, "colour": "lc", "permutation": IDENTITY, "factor": 1.0, "color_index": 1}],
         [{"process": 1, "colour": "lc", "permutation": [1, 0, 2, 3, 4], "factor": 1.0, "color_index": 1}],
         [{"process": 1, "colour": "lc", "permutation": IDENTITY, "factor": 0.25, "color_index": 1},
          {"process": 1, "colour": "lc", "permutation": [0, 1, 3, 2, 4], "factor": 0.75, "color_index": 1}]],
    ],
    "has_alpha_s": True, "has_color_flow": True,
}
CROSSING = [(0, 1.0), (1, 1.0), (2, 1.0), (4, 1.0), (3, 1.0)]  # qg>qgg: external leg l = input leg crossing[l]


def make_artifact(directory):
    """The artifact directory and its `.pacuda` file; returns the directory (absolute)."""
    d = os.path.abspath(directory)
    os.makedirs(d, exist_ok=True)
    f = pacuda_file.from_processes(NAMES, kernel=1, reference_points=0)
    f.processes[1].crossing = CROSSING
    pacuda_file.write(f, d + ".pacuda")
    return d


def events(count, stride, offset, seed=11, single=False):
    """Momenta as UMAMI lays them out (component k of particle l of event e at
    [e + stride * (LEGS * k + l)]), the point-major momenta of the events, channels and flavours
    (with `single`, only flavours of one contribution: helicity sampling takes no other)."""
    p = phase_space.sample(LEGS, count, seed)
    m = np.full(stride * LEGS * 4, np.nan)
    rows = m.reshape(LEGS * 4, stride)
    for k in range(4):
        for leg in range(LEGS):
            rows[LEGS * k + leg, offset:offset + count] = p[:, leg, k]
    rng = np.random.default_rng(seed)
    channel = np.zeros(stride, np.uint32)
    flavour = np.zeros(stride, np.int32)
    channel[offset:offset + count] = rng.integers(0, 2, count)
    for e in range(offset, offset + count):
        choices = [f for f, c in enumerate(SPEC["channels"][channel[e]]) if not single or len(c) == 1]
        flavour[e] = choices[rng.integers(0, len(choices))]
    return m, p, channel, flavour


_TEMPLATES = {}


def template(name):
    if name not in _TEMPLATES:
        _TEMPLATES[name] = processes.template(name)
    return _TEMPLATES[name]


def contribution_values(p, entry, oracle):
    """Per event (point-major p), the contribution's helicity values (f64, resolved from zero) of
    its process at its permuted (and crossed) momenta, from the oracle."""
    name = SPEC["processes"][entry["process"]]["key"]
    crossing = CROSSING if name == "qg>qgg" else [(l, 1.0) for l in range(LEGS)]
    q = np.empty_like(p)
    for l, (source, sign) in enumerate(crossing):
        q[:, l, :] = sign * p[:, entry["permutation"][source], :]
    _, out = oracle.evaluate(template(name), q, kernel=1)
    return out  # [event][helicity]


def expected(p, channel, flavour, offset, mode, oracle, alpha=None, random=None, helicity=None):
    """|M|^2, colour index and helicity label per event as the reference library computes them.
    Vectorised over events; every sum and draw runs over the helicities in order, so each value
    is the one the scalar arithmetic gives."""
    count = p.shape[0]
    ch = np.asarray(channel[offset:offset + count])
    fl = np.asarray(flavour[offset:offset + count])
    me, col, hel = np.zeros(count), np.zeros(count, np.int32), np.zeros(count, np.int32)
    cache = {}
    for c, channel_spec in enumerate(SPEC["channels"]):
        for f, sel in enumerate(channel_spec):
            ev = np.nonzero((ch == c) & (fl == f))[0]
            if ev.size == 0:
                continue
            vals = []
            for entry in sel:
                key = (entry["process"], tuple(entry["permutation"]))
                if key not in cache:
                    cache[key] = contribution_values(p, entry, oracle)
                t = template(SPEC["processes"][entry["process"]]["key"])
                num, den = t.meta["group_factor"]
                a0, power = t.meta["alpha_s"], t.meta["qcd_power"]
                a = np.full(ev.size, a0) if alpha is None else np.asarray(alpha[offset + ev], np.float64)
                scale = np.array([1.0 if x == a0 else math.pow(x / a0, power) for x in a])
                v = cache[key][ev].copy()
                live = np.array([t.offsets[h + 1] > t.offsets[h] for h in range(t.outputs)])
                if num != den:
                    v = v * float(num) / float(den)
                v = np.where(scale[:, None] != 1.0, v * scale[:, None], v)
                v[:, ~live] = 0.0
                vals.append((entry, v, live))
            first = sel[0]
            total = np.zeros(ev.size)
            label = np.zeros(ev.size, np.int32)
            if mode == "helicity":
                label = np.asarray(helicity[offset + ev], np.int32)
                for entry, v, _ in vals:
                    total = total + entry["factor"] * v[np.arange(ev.size), label]
            elif mode == "sample":
                _, v, live = vals[0]
                hs = np.nonzero(live)[0]
                s = np.zeros(ev.size)
                for h in hs:
                    s = s + v[:, h]
                target = np.asarray(random[offset + ev]) * s
                cumulative, pick, active = np.zeros(ev.size), np.zeros(ev.size, np.int32), np.ones(ev.size, bool)
                for h in hs:
                    take = active & (v[:, h] > 0.0)
                    pick = np.where(take, h, pick)
                    cumulative = np.where(take, cumulative + v[:, h], cumulative)
                    active = active & ~(take & (cumulative > target))
                total = s * first["factor"]
                label = pick
            else:
                for entry, v, _ in vals:
                    value = np.zeros(ev.size)
                    for h in range(v.shape[1]):
                        value = value + v[:, h]
                    total = total + entry["factor"] * value
            me[ev], col[ev], hel[ev] = total, first.get("color_index", 0), label
    return me, col, hel
