"""Deterministic test scenarios shared by the GPU worker (which runs them on a runner library in
a fresh process per kernel kind) and the tests (which run the same scenarios on the oracle).

A scenario is a plan call with every current and amplitude plane uploaded from seeded values and
every plane downloaded, so that a run's whole effect on the arena is compared; or a physics plan
evaluated at seeded RAMBO points with its amplitudes downloaded and its resolved reduction.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pacuda_b200 import abi, phase_space, plan as P, processes  # noqa: E402


def random_rows(rng, planes, amps, forms, scales, factors, rows=60):
    """Valid random rows exercising every op: sources first; contribution runs (one op per
    destination run); propagators, identities, clears and closures interleaved."""
    out = []
    for _ in range(int(rng.integers(1, 5))):
        family = int(rng.integers(0, 4))
        orientation = int(rng.integers(0, 2)) if family in (1, 2) else 0
        h = int(rng.choice([-1, 1]))
        ch = int(rng.choice([-1, 1])) if family == 1 else 0
        mass_slot = int(rng.integers(0, scales))
        out.append((12, int(rng.integers(0, planes - 4)), int(rng.integers(0, forms)), int(rng.integers(0, factors)),
                    mass_slot, P.source_code(family, orientation, h, ch)))
    while len(out) < rows:
        kind = rng.random()
        if kind < 0.55:
            op = int(rng.integers(2, 7))
            c0, c1, cd = P.contribution_shape(op)
            dst = int(rng.integers(0, planes - cd))
            # a destination's run has one op: a run whose component count changes reads sums the
            # reference runner never initialised (its `acc` registers), so such plans are invalid
            if out and out[-1][0] in (2, 3, 4, 5, 6) and out[-1][5] == dst and out[-1][0] != op:
                continue
            for k in range(int(rng.integers(1, 4))):
                out.append((op, int(k == 0 and rng.random() < 0.7), int(rng.integers(0, scales)),
                            int(rng.integers(0, planes - c0)), int(rng.integers(0, planes - c1)), dst,
                            int(rng.integers(0, forms)), int(rng.integers(0, forms)), int(rng.integers(0, factors))))
        elif kind < 0.7:
            op = int(rng.integers(7, 10))
            m = 4 if op == 9 else 2
            out.append((op, int(rng.integers(0, planes - m)), int(rng.integers(0, forms)), int(rng.integers(0, factors))))
        elif kind < 0.78:
            n = int(rng.integers(1, 7))
            out.append((10, int(rng.integers(0, planes - n)), n, int(rng.integers(0, factors))))
        elif kind < 0.83:
            n = int(rng.integers(1, 5))
            out.append((1, int(rng.integers(0, planes - n)), n))
        else:
            n = int(rng.integers(1, 5))
            out.append((11, int(rng.integers(0, planes - n)), int(rng.integers(0, planes - n)), int(rng.integers(0, amps)),
                        int(rng.integers(0, factors)), int(rng.integers(0, factors - n)), n))
    return out


def fuzz_case(seed, points=37, stride=40):
    """A random plan with all planes uploaded and downloaded; forms uploaded (seed even) or built
    on the device from external momenta (seed odd)."""
    rng = np.random.default_rng(1000 + seed)
    planes, amps, forms, scales, factors = 48, 5, 6, 3, 10
    rows = random_rows(rng, planes, amps, forms, scales, factors)
    width = P.widths_for(rows, planes, amps, forms, factors, scales, k_max=7)
    words = P.encode(rows, width)
    cre = rng.uniform(-1, 1, planes * stride)
    cim = rng.uniform(-1, 1, planes * stride)
    are = rng.uniform(-1, 1, amps * stride)
    aim = rng.uniform(-1, 1, amps * stride)
    kw = dict(words=words, width=width, stride=stride, points=points, current_planes=planes, amplitude_planes=amps,
              momentum_planes=4 * forms, scales=(rng.uniform(-0.6, 0.6, scales), rng.uniform(-0.6, 0.6, scales)),
              factors=(rng.uniform(-0.6, 0.6, factors), rng.uniform(-0.6, 0.6, factors)),
              upload_current=upload_runs(rows, planes), upload_amplitude=[0, amps - 1], zero_amplitude=[amps - 1, 1],
              download_amplitude=[0, amps], download_current=[0, planes], words_key=0,
              current=(cre, cim), amplitude=(are, aim))
    ext = None
    if seed % 2 == 0:
        mom = np.zeros(4 * forms * stride)
        for f in range(forms):
            for k in range(4):
                mom[(4 * f + k) * stride:(4 * f + k + 1) * stride] = (
                    rng.uniform(2.0, 3.0, stride) if k == 0 else rng.uniform(-1.5, 1.5, stride))
        kw["momenta"] = mom
    else:
        legs = 4
        ext = rng.uniform(-2, 2, legs * 4 * points)
        terms, slots, coef = [], [], []
        for f in range(forms):
            n = int(rng.integers(1, 3))  # an empty form is a null momentum: 1 / k^2 is infinite
            terms += [len(slots), n]
            for leg in rng.choice(legs, n, replace=False):  # distinct legs: no cancelling terms
                slots.append(int(leg))
                coef.append(float(rng.choice([-1.0, 1.0, 0.5])))
        kw.update(external=ext, external_count=legs, form_terms=terms, term_slots=slots, term_coefficients=coef,
                  flags=abi.FORMS_ON_DEVICE, momenta=np.zeros(4 * forms * stride))
    return kw


def upload_runs(rows, planes):
    """Every plane but those the plan's source rows write, as (first, count) runs: a call does not
    upload what its own sources compute (the reference converts such an upload after the sources
    ran, which is not a meaningful call)."""
    written = np.zeros(planes, dtype=bool)
    for r in rows:
        if r[0] == 12:
            n = 1 if r[5] & 7 == 0 else 2 if r[5] & 7 == 1 else 4
            written[r[1]:r[1] + n] = True
    runs, p = [], 0
    while p < planes:
        if written[p]:
            p += 1
            continue
        q = p
        while q < planes and not written[q]:
            q += 1
        runs += [p, q - p]
        p = q
    return runs


def fuzz_args(seed):
    """The CallArgs of fuzz case `seed` (fresh copies of its arrays)."""
    kw = fuzz_case(seed)
    return abi.CallArgs(**kw)


FUZZ_SEEDS = list(range(24))
PHYSICS = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g", "gg>gg", "q~g>q~gg"]


def physics_points(name, points=64, seed=11):
    legs = processes.PROCESSES[name]
    return phase_space.sample(len(legs), points, seed)


def source_cases(n=600, seed=3):
    """Template codes, masses and momenta for every family, orientation, helicity and chirality,
    both energy signs, with transverse-momentum-free and zero-momentum edge cases (as the
    reference's tests/check_sources.py draws them)."""
    rng = np.random.default_rng(seed)
    codes, masses, moms = [], [], []
    fams = [(0, 0, [0], [0], [0.0]), (1, 0, [-1, 1], [-1, 1], [0.0]), (1, 1, [-1, 1], [-1, 1], [0.0]),
            (2, 0, [-1, 1], [0], [0.0, 4.7, 91.188, 1e-9]), (2, 1, [-1, 1], [0], [0.0, 4.7, 173.0]),
            (3, 0, [-1, 1], [0], [0.0]), (3, 0, [-1, 0, 1], [0], [80.4, 91.188])]
    per = n // len(fams)
    for family, orientation, hs, chs, ms in fams:
        for _ in range(per):
            m = float(rng.choice(ms))
            kind = rng.random()
            if kind < 0.15:
                p3 = [0.0, 0.0, float(rng.choice([-1, 1])) * rng.uniform(1, 500)]
            elif kind < 0.2:
                p3 = [0.0, 0.0, 0.0]
            else:
                p3 = list(rng.uniform(-500, 500, 3))
            e = float(np.sqrt(sum(x * x for x in p3) + m * m))
            if e == 0.0:
                e = 1.0
            sgn = float(rng.choice([1.0, -1.0]))
            moms.append([sgn * e] + [sgn * x for x in p3])
            codes.append(P.source_code(family, orientation, int(rng.choice(hs)), int(rng.choice(chs))))
            masses.append(m)
    return np.array(codes, dtype=np.uint32), np.array(masses), np.array(moms).reshape(-1)
