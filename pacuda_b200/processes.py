"""Berends-Giele recurrence plans for massless QCD processes, in the runner's word format.

No `.pacuda` file ships with the reference (its converter needs MadGraph7 and RustiCol), so the
plans the runner executes are generated here. A plan computes, per phase-space point, every
leading-colour colour-ordered amplitude of a process for every helicity configuration, from
off-shell currents built by the Berends-Giele recursion:

* gluon currents J(w) for ordered words w of gluon legs: three-gluon vertices (op 6) over every
  split w = u v, the four-gluon vertex through an antisymmetric-tensor auxiliary current
  T(w) = sum over splits of J(u) ^ J(v) (op 5), contracted back into vectors (op 4), then the
  Feynman-gauge propagator (op 9);
* quark currents psi(q w) (two-component Weyl spinors) along the one quark line: the
  quark-gluon vertex (ops 2/3) over every split, then the Weyl propagator (ops 7/8);
* external wavefunctions by op 12 source rows; every amplitude is a closure (op 11) of the
  un-propagated closing current with the closing leg's wavefunction.

The rows are emitted stage by stage (stage = number of legs of a current) and, within a stage,
grouped by executor (op 6, ops 2/3, op 5, op 4, then the propagators), as RustiCol lays out a
Direct-Arena plan (rusticol/patches/0004: one row group per executor and stage). Couplings are
scale slots; signs and phases are exact factors.

Colour: the reduction weights are the leading-colour diagonal weights, N^(n-2) (N^2 - 1) per
gluon ordering (times 2 for the reflection partner that is not computed) and N^(k-1) (N^2 - 1)
per ordering of k gluons on a quark line. The process-group factor holds the spin and colour
averages and the identical-particle factor. Four-quark processes need a spinor-bilinear vector
current that no intrinsic op provides (the reference runs such executors as symjit rows, op 13),
so they are outside this generator.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass

import numpy as np

from . import plan as P

N_C = 3.0
ALPHA_S = 0.118


@dataclass(frozen=True)
class Leg:
    kind: str        # "g", "q" (quark) or "qb" (antiquark), as the physical particle
    incoming: bool


# Phases and signs of the vertices. The three-gluon coupling multiplies op 6's bracket
# (l.r)(u - v) + 2((l.v) r - (r.u) l); the four-gluon coupling multiplies op 4 of the tensor
# T(u) = J(x) ^ J(y) against J(v), with opposite signs for T on the left or right of the split;
# the quark-gluon coupling multiplies ops 2/3. The values are pinned by the Parke-Taylor and
# MHV tests (tests/test_physics.py).
G3 = 1j / math.sqrt(2.0)
G4 = 0.5j
# The quark line: per chirality (the outgoing-picture helicity of the line's quark end) the
# vertex and propagator ops. A line alternates the two Weyl matrices (ops 2/7 share one, 3/8
# the other), so its vertex and propagator are of different types. The closure contracts the
# closing current with the antiquark end's spinor component by component.
QUARK_OPS = {+1: (2, 8), -1: (3, 7)}
GQ = 1.0 / math.sqrt(2.0)
QUARK_CLOSE = (1.0, 1.0)

class Builder:
    def __init__(self):
        self.planes = 0
        self.forms = {}        # frozenset of legs -> form index
        self.form_list = []
        self.factors = {}      # complex -> index
        self.factor_list = []
        self.scales = []
        self.sources = []
        self.stage_rows = {}   # stage -> {group: [rows]}
        self.closures = []
        self.amplitudes = 0

    def plane(self, n):
        p = self.planes
        self.planes += n
        return p

    def form(self, legs):
        key = frozenset(legs)
        if key not in self.forms:
            self.forms[key] = len(self.form_list)
            self.form_list.append(sorted(key))
        return self.forms[key]

    def factor(self, z):
        z = complex(z)
        if z not in self.factors:
            self.factors[z] = len(self.factor_list)
            self.factor_list.append(z)
        return self.factors[z]

    def factor_run(self, zs):
        """A run of consecutive factor entries (closure component factors)."""
        zs = [complex(z) for z in zs]
        for start in range(len(self.factor_list) - len(zs) + 1):
            if self.factor_list[start:start + len(zs)] == zs:
                return start
        start = len(self.factor_list)
        for z in zs:
            self.factors.setdefault(z, len(self.factor_list))
            self.factor_list.append(z)
        return start

    def scale(self, z):
        self.scales.append(complex(z))
        return len(self.scales) - 1

    def add(self, stage, group, row):
        self.stage_rows.setdefault(stage, {}).setdefault(group, []).append(row)

    def rows(self):
        out = list(self.sources)
        order = ["vertex3", "quark", "wedge", "tensor", "prop", "qprop"]
        for stage in sorted(self.stage_rows):
            groups = self.stage_rows[stage]
            for g in order:
                out.extend(groups.get(g, []))
        out.extend(self.closures)
        return out


def _signs(legs):
    return [-1.0 if leg.incoming else 1.0 for leg in legs]


def outgoing_kind(leg):
    """The leg's kind in the all-outgoing picture (an incoming quark is an outgoing antiquark)."""
    if leg.kind == "g":
        return "g"
    if leg.incoming:
        return "qb" if leg.kind == "q" else "q"
    return leg.kind


def build(legs, alpha_s=ALPHA_S, gauge_leg=None, part=(0, 1)):
    """The plan (a `plan.Template`) of a process with these legs: all gluons, or one quark line
    (one outgoing-picture quark and one antiquark) and gluons.

    `gauge_leg`: a gluon leg whose wavefunction is left to the caller (no source row): the
    gauge-invariance test uploads its momentum there.
    `part`: (k, parts): only the colour orderings k, k + parts, ... (a process whose plan does not
    fit 64-bit words is split into parts, each its own plan; their outputs add up)."""
    n = len(legs)
    kinds = [outgoing_kind(leg) for leg in legs]
    gluons = [l for l in range(n) if kinds[l] == "g"]
    quarks = [l for l in range(n) if kinds[l] == "q"]
    antiquarks = [l for l in range(n) if kinds[l] == "qb"]
    if len(quarks) != len(antiquarks) or len(quarks) > 1:
        raise ValueError("one quark line at most: four-quark processes need symjit rows")
    g = math.sqrt(4.0 * math.pi * alpha_s)
    b = Builder()
    mass_slot = b.scale(0.0)
    s3 = b.scale(G3 * g)
    s_wedge = b.scale(1.0)
    s4 = b.scale(G4 * g * g)
    one = b.factor(1.0)
    plus4 = b.factor(1.0)
    minus4 = b.factor(-1.0)

    # sources: every leg, both helicities. Helicities here are the all-outgoing picture's. A
    # gluon's template carries the physical helicity (its E < 0 wavefunction flips it back,
    # CONVENTIONS.md:60); a Weyl spinor's template carries the outgoing-picture helicity itself
    # and the chirality its wavefunction keeps nonzero for that energy sign (:56-57).
    sign = _signs(legs)
    src = {}   # (leg, outgoing-picture helicity) -> plane base
    for l in range(n):
        f = b.form([l])
        for h in (-1, 1):
            phys = int(h * sign[l])
            if kinds[l] == "g":
                base = b.plane(4)
                src[(l, h)] = base
                if l != gauge_leg:
                    b.sources.append((12, base, f, one, mass_slot, P.source_code(3, 0, phys, 0)))
            else:
                base = b.plane(2)
                src[(l, h)] = base
                orientation = 0 if legs[l].kind == "q" else 1
                b.sources.append((12, base, f, one, mass_slot, P.source_code(1, orientation, h, int(h * sign[l]))))

    quark_line = bool(quarks)
    if quark_line:
        close_leg = antiquarks[0]
        q_leg = quarks[0]
        sq = b.scale(GQ * g)
        orderings = [tuple(p) for p in itertools.permutations(gluons)]
    else:
        close_leg = gluons[0]
        rest = gluons[1:]
        orderings = [tuple(p) for p in itertools.permutations(rest) if p[0] < p[-1]] if len(rest) > 1 else [tuple(rest)]

    orderings = orderings[part[0]::part[1]]
    # the gluon words: contiguous sub-words of every ordering; the full word of a gluon-only
    # ordering is the closing current (no propagator, no tensor)
    full = set(orderings) if not quark_line else set()
    words = set()
    for o in orderings:
        for i in range(len(o)):
            for j in range(i + 1, len(o) + 1):
                words.add(o[i:j])
    words = sorted(words, key=lambda w: (len(w), w))
    hel_of = lambda w: list(itertools.product((-1, 1), repeat=len(w)))
    J = {}   # (word, helicities) -> base
    T = {}
    for l in gluons:
        for h in (-1, 1):
            J[((l,), (h,))] = src[(l, h)]
    max_len = max((len(w) for w in words), default=0)
    # tensor currents are needed for words that are proper sub-words of a longer gluon word
    need_tensor = set()
    for w in words:
        for i in range(len(w)):
            for j in range(i + 1, len(w) + 1):
                u = w[i:j]
                if 2 <= len(u) < len(w):
                    need_tensor.add(u)
    for w in words:
        if len(w) == 1:
            continue
        stage = len(w)
        closing = w in full
        for hs in hel_of(w):
            hmap = dict(zip(w, hs))
            base = b.plane(4)
            J[(w, hs)] = base
            first = True
            for k in range(1, len(w)):
                u, v = w[:k], w[k:]
                hu, hv = tuple(hmap[x] for x in u), tuple(hmap[x] for x in v)
                b.add(stage, "vertex3", (6, 1 if first else 0, s3, J[(u, hu)], J[(v, hv)], base,
                                         b.form(u), b.form(v), one))
                first = False
            for k in range(1, len(w)):
                u, v = w[:k], w[k:]
                hu, hv = tuple(hmap[x] for x in u), tuple(hmap[x] for x in v)
                if len(u) >= 2:
                    b.add(stage, "tensor", (4, 0, s4, T[(u, hu)], J[(v, hv)], base, 0, 0, plus4))
                if len(v) >= 2:
                    b.add(stage, "tensor", (4, 0, s4, T[(v, hv)], J[(u, hu)], base, 0, 0, minus4))
            if not closing:
                b.add(stage, "prop", (9, base, b.form(w), one))
        if w in need_tensor:
            for hs in hel_of(w):
                hmap = dict(zip(w, hs))
                base = b.plane(6)
                T[(w, hs)] = base
                for k in range(1, len(w)):
                    u, v = w[:k], w[k:]
                    hu, hv = tuple(hmap[x] for x in u), tuple(hmap[x] for x in v)
                    b.add(stage, "wedge", (5, 1 if k == 1 else 0, s_wedge, J[(u, hu)], J[(v, hv)], base, 0, 0, one))

    amplitudes = []   # (ordering, full helicity tuple by leg) -> amplitude plane
    amp_index = {}
    if quark_line:
        # quark currents psi(q w) for the prefixes w of every ordering (w may be empty)
        prefixes = sorted({o[:j] for o in orderings for j in range(0, len(o) + 1)}, key=lambda w: (len(w), w))
        Q = {}
        for hq in (-1, 1):
            Q[((), hq, ())] = src[(q_leg, hq)]
        vertex_of = QUARK_OPS
        for w in prefixes:
            if not w:
                continue
            stage = len(w) + 1
            closing = len(w) == len(gluons)
            for hq in (-1, 1):
                vop, pop = vertex_of[hq]
                for hs in hel_of(w):
                    hmap = dict(zip(w, hs))
                    base = b.plane(2)
                    Q[(w, hq, hs)] = base
                    for k in range(0, len(w)):
                        u, v = w[:k], w[k:]
                        hu, hv = tuple(hmap[x] for x in u), tuple(hmap[x] for x in v)
                        b.add(stage, "quark", (vop, 1 if k == 0 else 0, sq, Q[(u, hq, hu)], J[(v, hv)], base,
                                               0, 0, one))
                    if not closing:
                        b.add(stage, "qprop", (pop, base, b.form((q_leg,) + w), one))
        for o in orderings:
            for hq in (-1, 1):
                first = b.factor_run(QUARK_CLOSE)
                hqb = -hq
                for hs in hel_of(o):
                    a = b.amplitudes
                    b.amplitudes += 1
                    hel = {q_leg: hq, close_leg: hqb, **dict(zip(o, hs))}
                    out = tuple(hel[l] for l in range(n))
                    b.closures.append((11, Q[(o, hq, hs)], src[(close_leg, hqb)], a, one, first, 2))
                    amplitudes.append((o, out, a))
    else:
        first = b.factor_run((1.0, -1.0, -1.0, -1.0))
        for o in orderings:
            for hs in hel_of(o):
                hmap = dict(zip(o, hs))
                for h0 in (-1, 1):
                    a = b.amplitudes
                    b.amplitudes += 1
                    hel = {close_leg: h0, **hmap}
                    out = tuple(hel[l] for l in range(n))
                    b.closures.append((11, J[(o, hs)], src[(close_leg, h0)], a, one, first, 4))
                    amplitudes.append((o, out, a))

    rows = b.rows()
    # the reduction: one output per helicity configuration (all 2^n, in lexicographic order of
    # the legs' helicities; the ones no amplitude reaches have no planes)
    helicities = list(itertools.product((-1, 1), repeat=n))
    by_hel = {h: [] for h in helicities}
    k_glu = len(gluons)
    if quark_line:
        weight = N_C ** (k_glu - 1) * (N_C * N_C - 1.0)
    else:
        weight = N_C ** (n - 2) * (N_C * N_C - 1.0) * (2.0 if n > 3 else 1.0)
    for o, out, a in amplitudes:  # outputs are keyed by the physical helicities
        by_hel[physical_helicities(kinds, sign, out)].append(a)
    offsets, planes, weights = [0], [], []
    for h in helicities:
        for a in by_hel[h]:
            planes.append(a)
            weights.append(weight)
        offsets.append(len(planes))
    width = P.widths_for(rows, b.planes, b.amplitudes, len(b.form_list), len(b.factor_list), len(b.scales),
                         k_max=4)
    words = P.encode(rows, width)
    form_terms, term_slots, term_coefficients = [], [], []
    for legs_of in b.form_list:
        form_terms += [len(term_slots), len(legs_of)]
        for l in legs_of:
            term_slots.append(l)
            term_coefficients.append(sign[l])
    num, den = group_factor(legs)
    return P.Template(
        words=words, width=width, current_planes=b.planes, amplitude_planes=b.amplitudes,
        momentum_planes=4 * len(b.form_list),
        scale_re=np.array([z.real for z in b.scales]), scale_im=np.array([z.imag for z in b.scales]),
        factor_re=np.array([z.real for z in b.factor_list]), factor_im=np.array([z.imag for z in b.factor_list]),
        zero_amplitude=np.array([0, b.amplitudes], dtype=np.uint32),
        download_amplitude=np.array([0, b.amplitudes], dtype=np.uint32),
        external_count=n, form_terms=np.array(form_terms, dtype=np.uint32),
        term_slots=np.array(term_slots, dtype=np.uint32), term_coefficients=np.array(term_coefficients),
        offsets=np.array(offsets, dtype=np.uint32), planes=np.array(planes, dtype=np.uint32),
        weights=np.array(weights),
        meta={"legs": [(leg.kind, leg.incoming) for leg in legs], "orderings": orderings,
              "amplitudes": amplitudes, "helicities": helicities, "group_factor": (num, den),
              "alpha_s": alpha_s, "qcd_power": n - 2, "rows": len(rows)})


def physical_helicities(kinds, sign, out):
    """The physical helicities of an amplitude's outgoing-picture labels: a crossed leg's
    helicity flips."""
    return tuple(int(h * s) for h, s in zip(out, sign))


def group_factor(legs):
    """(numerator, denominator): the initial-state spin and colour averages and the
    identical-final-state factor."""
    den = 1
    for leg in legs:
        if leg.incoming:
            den *= 2 * (8 if leg.kind == "g" else 3)
    finals = {}
    for leg in legs:
        if not leg.incoming:
            finals[leg.kind] = finals.get(leg.kind, 0) + 1
    for count in finals.values():
        den *= math.factorial(count)
    return 1, den


PROCESSES = {
    # name: legs (incoming first)
    "gg>gg": [Leg("g", True), Leg("g", True), Leg("g", False), Leg("g", False)],
    "gg>ggg": [Leg("g", True), Leg("g", True), Leg("g", False), Leg("g", False), Leg("g", False)],
    "gg>gggg": [Leg("g", True), Leg("g", True)] + [Leg("g", False)] * 4,
    "qg>qgg": [Leg("q", True), Leg("g", True), Leg("q", False), Leg("g", False), Leg("g", False)],
    "qq~>ggg": [Leg("q", True), Leg("qb", True), Leg("g", False), Leg("g", False), Leg("g", False)],
    "q~g>q~gg": [Leg("qb", True), Leg("g", True), Leg("qb", False), Leg("g", False), Leg("g", False)],
    "gq>qgg": [Leg("g", True), Leg("q", True), Leg("q", False), Leg("g", False), Leg("g", False)],
    "gg>qq~g": [Leg("g", True), Leg("g", True), Leg("q", False), Leg("qb", False), Leg("g", False)],
    "qq~>gg": [Leg("q", True), Leg("qb", True), Leg("g", False), Leg("g", False)],
    "qg>qggg": [Leg("q", True), Leg("g", True), Leg("q", False)] + [Leg("g", False)] * 3,
    "qq~>gggg": [Leg("q", True), Leg("qb", True)] + [Leg("g", False)] * 4,
    "gg>qq~gg": [Leg("g", True), Leg("g", True), Leg("q", False), Leg("qb", False), Leg("g", False), Leg("g", False)],
}

# p p -> 3 jets: the subprocess families the intrinsic ops express (one quark line at most)
PP3J = ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"]
PP4J = ["gg>gggg", "qg>qggg", "qq~>gggg", "gg>qq~gg"]


def template(name, **kw):
    return build(PROCESSES[name], **kw)


def parts(name):
    """The fewest parts (1, 2, 3, 4, 6, ...) whose plans all fit 64-bit words: [template, ...].
    A part evaluates a subset of the colour orderings; the process's outputs are their sum."""
    for n in (1, 2, 3, 4, 5, 6, 8, 10, 12):
        try:
            return [template(name, part=(k, n)) for k in range(n)]
        except ValueError as e:
            if "bits" not in str(e):
                raise
    raise ValueError(f"{name}: no split into 12 or fewer parts fits 64-bit words")
