"""The on-chip executor's schedule, checked on the CPU: tasks, levels, slots and write-backs give
every plane and amplitude the value the reference's row order gives (symbolically; see
tests/schedule_emulator.py), for random plans and the physics plans."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

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


def _oracle_program(words, width):
    """The oracle's rows (the reference's decode and sort by destination) as instructions in the
    emulator's form, with F_FIRST / F_LAST around each destination's run of rows."""
    rows = [[int(v) for v in r] for r in O.decode(words, width, sort=True)]

    def dst_at(k):
        return rows[k][5] if 0 <= k < len(rows) and 2 <= rows[k][0] <= 6 else None

    prog = []
    for n, (op, *f) in enumerate(rows):
        if 2 <= op <= 6:
            flags = (E.F_INIT if f[0] else 0) | (E.F_FIRST if dst_at(n - 1) != f[4] else 0) | \
                    (E.F_LAST if dst_at(n + 1) != f[4] else 0)
            prog.append([E.K_CONTRIB | op << 4 | flags << 8, f[2], f[3], f[4],
                         (f[5] & 0xFFFF) | (f[6] << 16) if op == 6 else 0, f[1], f[7], 0])
        elif op == 1:
            prog.append([E.K_CLEAR | 1 << 4, f[0], f[1], 0, 0, 0, 0, 0])
        elif 7 <= op <= 9:
            prog.append([E.K_PROP | op << 4, f[0], 0, 0, f[1], 0, f[2], 0])
        elif op == 10:
            prog.append([E.K_IDENTITY | 10 << 4, f[0], f[1], 0, 0, 0, f[2], 0])
        elif op == 11:
            prog.append([E.K_CLOSURE | 11 << 4, f[0], f[1], f[2], 0, f[5], f[3], f[4]])
        else:
            prog.append([E.K_SOURCE | 12 << 4, f[0], 0, 0, f[1], f[3], f[2], f[4]])
    return np.array(prog, dtype=np.uint32).reshape(-1, 8)


def _grouping_case(words, width, planes, amps, forms, scales, factors):
    prog = E.export(words, width, planes, amps, forms, scales, factors)[0]
    want = E.reference(_oracle_program(words, width), planes, amps)
    assert E.reference(prog, planes, amps) == want
    # each destination of a contribution run is one F_FIRST .. F_LAST run of rows
    return prog


@pytest.mark.parametrize("seed", S.FUZZ_SEEDS)
def test_grouped_runs_give_the_sorted_values_random(seed):
    """The product gathers a contribution run's rows per destination at its first row, the
    reference sorts them by destination (recurrence_runner.cu:980-1007): every plane and amplitude
    gets the same operations on the same operands in the same order (symbolic values equal)."""
    kw = S.fuzz_case(seed)
    _grouping_case(kw["words"], kw["width"], kw["current_planes"], kw["amplitude_planes"],
                   kw["momentum_planes"] // 4, len(kw["scales"][0]), len(kw["factors"][0]))


@pytest.mark.parametrize("name", ["gg>ggg", "qg>qgg", "qq~>ggg", "gg>qq~g"])
def test_grouped_runs_give_the_sorted_values_physics(name):
    t = processes.template(name)
    prog = _grouping_case(t.words, t.width, t.current_planes, t.amplitude_planes, t.momentum_planes // 4,
                          len(t.scale_re), len(t.factor_re))
    # the grouping made every destination's rows one run: as many F_FIRST rows as destinations per run
    first = [(int(r[3]), bool((int(r[0]) >> 8) & E.F_FIRST)) for r in prog if int(r[0]) & 15 == E.K_CONTRIB]
    sorted_rows = O.decode(t.words, t.width, sort=True)
    runs_ref = sum(1 for k, r in enumerate(sorted_rows) if 2 <= r[0] <= 6 and
                   (k == 0 or not 2 <= sorted_rows[k - 1][0] <= 6 or sorted_rows[k - 1][5] != r[5]))
    assert sum(f for _, f in first) == runs_ref


def test_decode_status_codes():
    """Ops 0 and 15 and widths above 32 bits are INVALID (2); a symjit binding whose codes run
    past the last word is refused like every symjit row (3, as a runner without symjit kernels)."""
    lib = E.lib()
    lib.program_status.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p] + [C.c_uint32] * 5

    def status(words, width=(8, 8, 8, 8, 8, 8, 0, 0)):
        w = np.ascontiguousarray(words, dtype=np.uint64)
        wd = np.ascontiguousarray(width, dtype=np.uint8)
        return lib.program_status(w.ctypes.data, len(w), wd.ctypes.data, 64, 8, 8, 8, 8)

    assert status([0]) == 2 and status([15]) == 2
    assert status([1], width=(33, 8, 8, 8, 8, 8, 0, 0)) == 2
    assert status([14 | 3 << 20]) == 3  # three input codes, no data words
    assert status([1 | 2 << 4 | 3 << 12]) == 0  # clear planes 2..4
