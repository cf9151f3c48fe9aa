"""CPU tests of the oracle, the plan generator and the library boundary (no GPU needed)."""
import ctypes as C
import os
import re
from fractions import Fraction

import numpy as np
import pytest

from tests import scenarios as S
from oracle import oracle as O
from pacuda_b200 import abi, phase_space, plan as P, processes

ROOT = S.ROOT
G2 = 4 * np.pi * processes.ALPHA_S


def test_sources_match_reference_legend():
    """The oracle's wavefunctions against the reference's legend (tests/golden/sources_legend.npz,
    made by tests/golden/make_sources_golden.py from the reference's tests/check_sources.py): at
    most 1e-13 relative, that file's bar."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "sources_legend.npz"))
    got = O.sources(g["codes"], g["masses"], g["momenta"].reshape(-1))
    want = g["values"]
    scale = np.maximum(1e-300, np.abs(want).max(axis=1))
    err = np.abs(got - want).max(axis=1) / scale
    assert err.max() < 1e-13, dict(zip(g["names"][err >= 1e-13][:5], err[err >= 1e-13][:5]))
    # every family and both energy signs were exercised
    assert len(set(g["names"])) == 7 and (g["momenta"][:, 0] < 0).any() and (g["momenta"][:, 0] > 0).any()


def _s(k, i, j, pt):
    a = k[pt, i] + k[pt, j]
    return abs(a[0] ** 2 - a[1] ** 2 - a[2] ** 2 - a[3] ** 2)


@pytest.mark.parametrize("name", ["gg>gg", "gg>ggg", "qq~>gg", "qq~>ggg", "qg>qgg", "gg>qq~g", "q~g>q~gg", "gq>qgg"])
def test_amplitudes_match_mhv_formulas(name):
    """Known answers independent of the reference: every nonzero tree amplitude of these
    processes is MHV or anti-MHV, |A|^2 = g^2(n-2) s_ij^4 / prod s_adjacent for gluons (Parke,
    Taylor) and s_fi^3 s_(f-bar)i / prod s_adjacent for one quark line (f the fermion, i the gluon
    with the odd helicity); all other helicity amplitudes vanish."""
    legs = processes.PROCESSES[name]
    n = len(legs)
    t = processes.template(name)
    p = phase_space.sample(n, 3, 5)
    amps, _ = O.evaluate(t, p)
    sign = np.array([-1.0 if l.incoming else 1.0 for l in legs])
    k = p * sign[None, :, None]
    kinds = [processes.outgoing_kind(l) for l in legs]
    quark = "q" in kinds
    checked, worst, zero = 0, 0.0, 0.0
    for o, hel, a in t.meta["amplitudes"]:
        neg = [l for l in range(n) if hel[l] == -1]
        pos = [l for l in range(n) if hel[l] == 1]
        sel = neg if len(neg) == 2 else pos if len(pos) == 2 else None
        cyc = ([kinds.index("qb"), kinds.index("q")] if quark else [0]) + list(o)
        for pt in range(p.shape[0]):
            a2 = abs(amps[a, pt]) ** 2 / G2 ** (n - 2)
            if sel is None or (quark and sum(kinds[x] != "g" for x in sel) != 1):
                zero = max(zero, a2)
                continue
            den = np.prod([_s(k, cyc[m], cyc[(m + 1) % n], pt) for m in range(n)])
            if quark:
                f = [x for x in sel if kinds[x] != "g"][0]
                i = [x for x in sel if kinds[x] == "g"][0]
                fb = kinds.index("q") if kinds[f] == "qb" else kinds.index("qb")
                want = _s(k, f, i, pt) ** 3 * _s(k, fb, i, pt) / den
            else:
                want = _s(k, sel[0], sel[1], pt) ** 4 / den
            worst = max(worst, abs(a2 / want - 1))
            checked += 1
    assert checked > 0 and worst < 1e-11, worst
    typical = np.abs(amps).max() ** 2 / G2 ** (n - 2)
    assert zero < 1e-20 * max(typical, 1.0)


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg", "gg>qq~g"])
def test_amplitudes_are_gauge_invariant(name):
    """A gluon polarisation replaced by its momentum gives zero (every gluon in turn)."""
    legs = processes.PROCESSES[name]
    n = len(legs)
    kinds = [processes.outgoing_kind(l) for l in legs]
    p = phase_space.sample(n, 2, 7)
    sign = np.array([-1.0 if l.incoming else 1.0 for l in legs])
    ref, _ = O.evaluate(processes.template(name), p)
    for g in [l for l in range(n) if kinds[l] == "g"]:
        t = processes.build(legs, gauge_leg=g)
        args = t.call(phase_space.source_major(p), 2)
        base = 0
        for l in range(n):
            for h in (-1, 1):
                if l == g:
                    for c in range(4):
                        args.cre[(base + c) * 2:(base + c + 1) * 2] = sign[l] * p[:, l, c]
                base += 4 if kinds[l] == "g" else 2
        assert O.run(args, kernel=1) == 0
        assert np.abs(args.are + 1j * args.aim).max() < 1e-10 * np.abs(ref).max()


def test_five_gluon_helicity_sum_matches_closed_form():
    """sum over helicities and the 24 orderings of |A|^2, from the plan's resolved outputs,
    against the closed form 2 sum_(i<j) s_ij^4 sum_sigma 1 / prod s_adjacent (all 5-gluon
    amplitudes are MHV or anti-MHV), times the plan's colour weight and g^6."""
    import itertools
    t = processes.template("gg>ggg")
    p = phase_space.sample(5, 4, 9)
    _, out = O.evaluate(t, p)
    k = p * np.array([-1, -1, 1, 1, 1.0])[None, :, None]
    w = processes.N_C ** 3 * (processes.N_C ** 2 - 1)
    for pt in range(4):
        num = sum(_s(k, i, j, pt) ** 4 for i in range(5) for j in range(i + 1, 5))
        den = sum(1.0 / np.prod([_s(k, c[m], c[(m + 1) % 5], pt) for m in range(5)])
                  for c in [(0,) + q for q in itertools.permutations(range(1, 5))])
        want = 2 * num * den * w * G2 ** 3
        assert abs(out[pt].sum() / want - 1) < 1e-11


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg"])
def test_oracle_kinds_agree_with_f64(name):
    """runner_variants.sh's tolerances: df64 within 1e-9, mixed and mixed64 within 1e-4 of the
    largest f64 value; here on physics plans' resolved outputs."""
    t = processes.template(name)
    p = phase_space.sample(len(processes.PROCESSES[name]), 32, 13)
    _, want = O.evaluate(t, p, kernel=abi.KERNEL_F64)
    scale = np.abs(want).max()
    for kind, tol in [(abi.KERNEL_DF64, 1e-9), (abi.KERNEL_MIXED, 1e-4), (abi.KERNEL_MIXED64, 1e-4)]:
        _, got = O.evaluate(t, p, kernel=kind)
        assert np.abs(got - want).max() / scale <= tol, kind


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def test_oracle_reductions_match_host_reduction():
    """rectest's known answer (runner/rectest.c:130-259): each reduction equals the host's
    `out += w fma(re, re, im im)` in order, bit for bit."""
    t = processes.template("qg>qgg")
    p = phase_space.sample(5, 8, 3)
    n = 8
    args = t.call(phase_space.source_major(p), n)
    assert O.run(args, kernel=1) == 0
    out = np.linspace(0.25, 2.0, n * t.outputs)
    want = out.copy().reshape(n, t.outputs)
    for o in range(t.outputs):
        for i in range(n):
            v = want[i, o]
            for kk in range(t.offsets[o], t.offsets[o + 1]):
                at = int(t.planes[kk]) * n + i
                re_, im_ = args.are[at], args.aim[at]
                v = v + t.weights[kk] * _fma(re_, re_, im_ * im_)
            want[i, o] = v
    r, hold = abi.reduce_resolved_args(t.planes, t.weights, t.offsets, out, n, 1, t.outputs, 0)
    assert O.reduce_resolved(r, args.are, args.aim, n) == 0
    assert np.array_equal(out.reshape(n, t.outputs).view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg"])
def test_words_roundtrip_and_decode_like_the_runner(name):
    t = processes.template(name)
    rows = P.decode(t.words, t.width)
    assert np.array_equal(P.encode(rows, t.width), t.words)
    dec = O.decode(t.words, t.width, sort=False)
    assert len(dec) == len(rows)
    for r, d in zip(rows, dec):
        assert list(r) == list(d[: len(r)])


def test_fuzz_plans_run_on_every_oracle_kind():
    for seed in S.FUZZ_SEEDS[:6]:
        for kind in range(4):
            assert O.run(S.fuzz_args(seed), kernel=kind) == 0


def test_oracle_rejects_symjit_rows_and_bad_words():
    width = [8, 4, 4, 4, 2, 3, 0, 0]
    words = P.encode([(12, 0, 0, 0, 0, P.source_code(3, 0, 1, 0))], width)
    a = abi.CallArgs(words=np.concatenate([words, np.array([13], dtype=np.uint64)]), width=width, stride=4, points=4,
                     current=(np.zeros(40), np.zeros(40)), amplitude=(np.zeros(4), np.zeros(4)), current_planes=10,
                     amplitude_planes=1, momentum_planes=4, momenta=np.ones(16), scales=([0.0], [0.0]),
                     factors=([1.0], [0.0]))
    assert O.run(a, kernel=1) == abi.DEVICE_ERROR      # symjit rows: no kernels in this runner
    a.words[-1] = 0                                     # op 0 is no op
    assert O.run(a, kernel=1) == abi.INVALID


def test_phase_space_is_physical():
    p = phase_space.sample(5, 500, 1, ecm=13000.0)
    tot_in = p[:, 0] + p[:, 1]
    tot_out = p[:, 2:].sum(axis=1)
    assert np.allclose(tot_in, tot_out, atol=1e-8)
    m2 = p[..., 0] ** 2 - (p[..., 1:] ** 2).sum(axis=2)
    assert np.abs(m2).max() < 1e-6
    assert phase_space.passes_cuts(p).all()
    # a point can be regenerated alone
    q = phase_space.rambo(5, 3, 42, first=7)
    assert np.array_equal(q, phase_space.rambo(5, 10, 42)[7:10])


HEADER = os.path.join(ROOT, "include", "pacman_recurrence.h")
LIB = os.path.join(ROOT, "pacuda_b200", "librecurrence.so")


def test_library_loads_and_exports_every_declared_symbol():
    """The C-ABI library loads without a GPU and exports every function include/*.h declares."""
    from pacuda_b200 import build
    build.build()
    lib = C.CDLL(LIB)
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(pacman_recurrence_v1_\w+|pacuda_b200_\w+)\s*\(", text))
    assert "pacman_recurrence_v1_run" in names and len(names) >= 10
    for name in sorted(names):
        assert hasattr(lib, name), name


def test_surrogate_library_exports_every_declared_symbol():
    """libsurrogate.so loads without a GPU and exports every function include/pacuda_surrogate.h
    declares (no compute calls)."""
    from pacuda_b200 import build
    build.build()
    lib = C.CDLL(build.SG_LIB)
    text = open(os.path.join(ROOT, "include", "pacuda_surrogate.h")).read()
    names = set(re.findall(r"\b(pacuda_(?:sg|uw)_\w+)\s*\(", text))
    assert {"pacuda_sg_create", "pacuda_sg_train_step", "pacuda_sg_forward", "pacuda_uw_stage1"} <= names
    for name in sorted(names):
        assert hasattr(lib, name), name
    lib.pacuda_sg_param_count.restype = C.c_size_t
    assert lib.pacuda_sg_param_count() == 256 * 64 + 3 * 256 * 256 + 5 * 256 + 1


def test_abi_struct_layout_is_the_references():
    """The ctypes mirror has the reference's layout (runner/pacman_recurrence.h:18-138 on LP64, as
    gcc lays out both that header and include/pacman_recurrence.h)."""
    assert C.sizeof(abi.Call) == 248
    assert abi.CALL_V1_SIZE == 192 and abi.CALL_V2_SIZE == 208
    assert C.sizeof(abi.Reduce) == 40
    assert C.sizeof(abi.ReduceResolved) == 64
    assert C.sizeof(abi.ReduceSample) == 96
    assert C.sizeof(abi.Options) == 24


def test_six_gluon_parts_match_mhv_formulas_and_vanish():
    """gg>gggg, split into parts of its 60 colour orderings (one plan would not fit 64-bit words):
    every MHV and anti-MHV amplitude matches Parke-Taylor, every amplitude with at most one
    negative or one positive helicity vanishes (NMHV ones are covered by the gauge test below)."""
    legs = processes.PROCESSES["gg>gggg"]
    n = len(legs)
    parts = processes.parts("gg>gggg")
    assert len(parts) > 1 and sum(len(t.meta["orderings"]) for t in parts) == 60
    p = phase_space.sample(n, 2, 5)
    sign = np.array([-1.0 if l.incoming else 1.0 for l in legs])
    k = p * sign[None, :, None]
    checked, worst, zero, typical = 0, 0.0, 0.0, 0.0
    for t in parts:
        amps, _ = O.evaluate(t, p)
        typical = max(typical, np.abs(amps).max() ** 2 / G2 ** (n - 2))
        for o, hel, a in t.meta["amplitudes"]:
            neg = [l for l in range(n) if hel[l] == -1]
            pos = [l for l in range(n) if hel[l] == 1]
            cyc = [0] + list(o)
            for pt in range(p.shape[0]):
                a2 = abs(amps[a, pt]) ** 2 / G2 ** (n - 2)
                if len(neg) <= 1 or len(pos) <= 1:
                    zero = max(zero, a2)
                elif len(neg) == 2 or len(pos) == 2:
                    sel = neg if len(neg) == 2 else pos
                    den = np.prod([_s(k, cyc[m], cyc[(m + 1) % n], pt) for m in range(n)])
                    worst = max(worst, abs(a2 / (_s(k, sel[0], sel[1], pt) ** 4 / den) - 1))
                    checked += 1
    assert checked > 0 and worst < 1e-11, worst
    assert zero < 1e-20 * typical


def test_six_gluon_part_is_gauge_invariant():
    """A gluon polarisation replaced by its momentum zeroes every amplitude of a gg>gggg part,
    NMHV ones included."""
    legs = processes.PROCESSES["gg>gggg"]
    n = len(legs)
    nparts = len(processes.parts("gg>gggg"))
    p = phase_space.sample(n, 2, 7)
    sign = np.array([-1.0 if l.incoming else 1.0 for l in legs])
    ref, _ = O.evaluate(processes.template("gg>gggg", part=(1, nparts)), p)
    for g in (0, 3):
        t = processes.build(legs, gauge_leg=g, part=(1, nparts))
        args = t.call(phase_space.source_major(p), 2)
        for h in range(2):
            base = 4 * (2 * g + h)
            for c in range(4):
                args.cre[(base + c) * 2:(base + c + 1) * 2] = sign[g] * p[:, g, c]
        assert O.run(args, kernel=1) == 0
        assert np.abs(args.are + 1j * args.aim).max() < 1e-10 * np.abs(ref).max()
