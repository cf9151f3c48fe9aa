"""The on-chip executor's schedule, checked on the CPU: tasks, levels, slots and write-backs give
every plane and amplitude the value the reference's row order gives (symbolically; see
tests/schedule_emulator.py), for random plans and the physics plans."""
import numpy as np
import pytest

from tests import scenarios as S
from tests import schedule_emulator as E
from pacuda_b200 import processes


def check(words, width, planes, amps, forms, scales, factors):
    prog, ins, tf, lf, loads, ampp, slots, sources = E.export(words, width, planes, amps, forms, scales, factors)
    want = E.reference(prog, planes, amps)
    for reverse in (False, True):
        got = E.scheduled(ins, tf, lf, loads, ampp, slots, planes, amps, reverse=reverse)
        bad_c = [p for p in range(planes) if got[0][p] != want[0][p]]
        bad_a = [q for q in range(amps) if got[1][q] != want[1][q]]
        assert not bad_c and not bad_a, f"planes {bad_c[:10]} amplitudes {bad_a[:10]} (reverse={reverse})"


@pytest.mark.parametrize("seed", S.FUZZ_SEEDS)
def test_random_plans(seed):
    kw = S.fuzz_case(seed)
    check(kw["words"], kw["width"], kw["current_planes"], kw["amplitude_planes"], kw["momentum_planes"] // 4,
          len(kw["scales"][0]), len(kw["factors"][0]))


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg", "gg>qq~g"])
def test_physics_plans(name):
    t = processes.template(name)
    check(t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4, len(t.scale_re),
          len(t.factor_re))


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg", "gg>qq~g"])
def test_term_mode_gives_every_reduction_term_its_value(name):
    """Batch plans keep reduction terms instead of amplitudes (use_terms): every term is made from
    the same amplitude value as the reference's row order gives, for the physics plans (where it
    applies) and for a plan where an amplitude has two closure rows (where it must not)."""
    t = processes.template(name)
    args = (t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4, len(t.scale_re),
            len(t.factor_re))
    applied, ins, tf, lf, terms, slots = E.export_terms(*args, t.offsets, t.planes)
    assert applied and terms == len(t.planes)
    prog = E.export(*args)[0]
    want = E.reference_terms(prog, t.current_planes, t.amplitude_planes, t.planes)
    for reverse in (False, True):
        assert E.scheduled_terms(ins, tf, lf, slots, terms, t.current_planes, reverse=reverse) == want


def test_term_mode_refuses_shared_terms():
    t = processes.template("qg>qgg")
    args = (t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4, len(t.scale_re),
            len(t.factor_re))
    planes = np.concatenate([t.planes, t.planes[:1]])  # an amplitude in two terms
    offsets = np.concatenate([t.offsets, [t.offsets[-1] + 1]])
    applied = E.export_terms(*args, offsets, planes)[0]
    assert not applied


def test_six_gluon_part_plan():
    """A gg>gggg part (16-17 thousand rows, 5 levels, about 10 000 slots per point)."""
    t = processes.parts("gg>gggg")[0]
    check(t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4, len(t.scale_re),
          len(t.factor_re))


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg"])
def test_spread_slots(name):
    """The spread slot placement: every operand's slots lie in one window of 12 slots (the
    13th of each 13 is never used), and the 4-slot currents start in all eight 16-byte bank
    groups (slot mod 8)."""
    t = processes.template(name)
    args = (t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4, len(t.scale_re),
            len(t.factor_re))
    applied, ins, tf, lf, terms, slots = E.export_terms(*args, t.offsets, t.planes)
    shape = {2: (2, 4, 2), 3: (2, 4, 2), 4: (6, 4, 4), 5: (4, 4, 6), 6: (4, 4, 4)}
    starts = set()
    for row in ins:
        kind, op = int(row[0]) & 15, (int(row[0]) >> 4) & 15
        a, b, c = int(row[1]), int(row[2]), int(row[3])
        if kind != 1:
            continue
        c0, c1, cd = shape[op]
        for base, n in ((a, c0), (b, c1), (c, cd)):
            assert base // 13 == (base + n - 1) // 13 and (base + n - 1) % 13 != 12, (base, n)
            assert base + n <= slots
        if c1 == 4:
            starts.add(b % 8)
    assert starts == set(range(8))
