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
