"""A symbolic emulator of the on-chip executor's schedule (test infrastructure).

Every value is a token: a hash of the operation that made it and its operands' tokens. The
program is run once in the reference's order with the reference's semantics (F_FIRST/F_LAST
sums, in-place finalisations, closures into amplitudes), and once as the schedule runs it (levels
in order, the tasks of a level in reverse order, values in slots, live-in planes loaded, every
plane's last value written back, every amplitude stored at the end). The two final arenas must
hold the same tokens: then the schedule computes every value from the same operands in the
same order, whatever the arithmetic.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "harness")
LIB = os.path.join(HARNESS, "libschedule_harness.so")
K_CONTRIB, K_PROP, K_IDENTITY, K_CLEAR, K_CLOSURE, K_SOURCE = 1, 2, 3, 4, 5, 6
F_INIT, F_FIRST, F_LAST, F_WB, F_ACC0, F_NOSTORE, F_TERM = 1, 2, 4, 8, 16, 32, 64
ZERO = hash(("zero amplitude",))
_lib = None


def lib():
    global _lib
    if _lib is None:
        subprocess.run(["make", "-s", "-C", HARNESS], check=True)
        _lib = C.CDLL(LIB)
        sig = [C.c_void_p, C.c_uint32, C.c_void_p] + [C.c_uint32] * 5
        _lib.program_export.argtypes = sig + [C.c_void_p, C.c_void_p]
        _lib.schedule_export.argtypes = sig + [C.c_void_p] * 7
        _lib.schedule_stats.argtypes = sig + [C.c_void_p]
        _lib.schedule_export_terms.argtypes = sig + [C.c_void_p, C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
    return _lib


def _args(words, width, planes, amps, forms, scales, factors):
    words = np.ascontiguousarray(words, dtype=np.uint64)
    width = np.ascontiguousarray(list(width)[:8] + [0] * (8 - len(list(width)[:8])), dtype=np.uint8)
    return (words, width), [words.ctypes.data, len(words), width.ctypes.data, planes, amps, forms, scales, factors]


def stats(words, width, planes, amps, forms, scales, factors):
    keep, a = _args(words, width, planes, amps, forms, scales, factors)
    st = np.zeros(9, dtype=np.uint32)
    assert lib().schedule_stats(*a, st.ctypes.data) == 0
    return dict(zip(["instructions", "tasks", "levels", "cur_slots", "amp_slots", "max_task_len", "live_in_groups",
                     "max_tasks_per_level", "peak_live"], st.tolist()))


def export(words, width, planes, amps, forms, scales, factors):
    keep, a = _args(words, width, planes, amps, forms, scales, factors)
    n = np.zeros(1, dtype=np.uint32)
    assert lib().program_export(*a, n.ctypes.data, None) == 0
    prog = np.zeros(8 * int(n[0]), dtype=np.uint32)
    assert lib().program_export(*a, n.ctypes.data, prog.ctypes.data) == 0
    sizes = np.zeros(8, dtype=np.uint32)
    null = [None] * 7
    assert lib().schedule_export(*a, sizes.ctypes.data, *null) == 0
    ins = np.zeros(8 * int(sizes[0]) + 8, dtype=np.uint32)
    tf = np.zeros(int(sizes[1]) + 1, dtype=np.uint32)
    lf = np.zeros(int(sizes[2]) + 1, dtype=np.uint32)
    loads = np.zeros(int(sizes[3]) + 1, dtype=np.uint32)
    ampp = np.zeros(int(sizes[4]) + 1, dtype=np.uint32)
    assert lib().schedule_export(*a, sizes.ctypes.data, ins.ctypes.data, tf.ctypes.data, lf.ctypes.data,
                                 loads.ctypes.data, ampp.ctypes.data, None) == 0
    return (prog.reshape(-1, 8), ins[: 8 * int(sizes[0])].reshape(-1, 8), tf[: int(sizes[1])], lf[: int(sizes[2])],
            loads[: int(sizes[3])], ampp[: int(sizes[4])], int(sizes[5]), int(sizes[6]))


def _shape(op):
    c0 = 6 if op == 4 else 4 if op in (5, 6) else 2
    cd = 4 if op in (4, 6) else 6 if op == 5 else 2
    return c0, 4, cd


def _src_comps(code):
    f = code & 7
    return 1 if f == 0 else 2 if f == 1 else 4


def _head(i):
    h = int(i[0])
    return h & 15, (h >> 4) & 15, (h >> 8) & 255


class _Store:
    """Values by address: planes of the arena, or slots."""

    def __init__(self, get, put, amp_get, amp_put, term_put=None):
        self.get, self.put, self.amp_get, self.amp_put, self.term_put = get, put, amp_get, amp_put, term_put


def _row(store, i, acc, wb=None):
    kind, op, flags = _head(i)
    a, b, c, f, s, x, y = (int(v) for v in i[1:])
    if kind == K_CONTRIB:
        c0, c1, cd = _shape(op)
        l = tuple(store.get(a + k) for k in range(c0))
        r = tuple(store.get(b + k) for k in range(c1))
        forms = (f,) if op == 6 else ()
        for k in range(cd):
            val = hash(("contrib", op, s, x, l, r, forms, k))
            if not flags & F_FIRST:
                acc[k] = hash(("add", acc[k], val))
            elif flags & F_INIT:
                acc[k] = val
            else:
                acc[k] = hash(("add", store.get(c + k), val))
        if flags & F_LAST:
            if not flags & F_NOSTORE:
                for k in range(cd):
                    store.put(c + k, acc[k])
            if wb and flags & F_WB:
                wb(y, [acc[k] for k in range(cd)])
    elif kind == K_PROP:
        m = 4 if op == 9 else 2
        cur = tuple(store.get(a + k) for k in range(m))
        out = [hash(("prop", op, f, x, cur, k)) for k in range(m)]
        for k in range(m):
            store.put(a + k, out[k])
        if wb and flags & F_WB:
            wb(y, out)
    elif kind == K_IDENTITY:
        for k in range(b):
            v = hash(("identity", x, store.get(a + k)))
            store.put(a + k, v)
            if wb and flags & F_WB:
                wb(y + k, [v])
    elif kind == K_CLEAR:
        for k in range(b):
            store.put(a + k, 0)
            if wb and flags & F_WB:
                wb(y + k, [0])
    elif kind == K_CLOSURE:
        v = ZERO if flags & F_TERM else store.amp_get(c)
        for k in range(s):
            left = acc[k] if flags & F_ACC0 else store.get(a + k)
            v = hash(("closure", x, y + k, left, store.get(b + k), v))
        if flags & F_TERM:
            if c != 0xffff:
                store.term_put(c, v)
        else:
            store.amp_put(c, v)
    elif kind == K_SOURCE:
        out = [hash(("source", y, f, x, s, k)) for k in range(_src_comps(y))]
        for k, v in enumerate(out):
            store.put(a + k, v)
        if wb and flags & F_WB:
            wb(c, out)


def reference(prog, planes, amps):
    arena = [hash(("init", p)) for p in range(planes)]
    amp = [hash(("amp", q)) for q in range(amps)]
    st = _Store(arena.__getitem__, arena.__setitem__, amp.__getitem__, amp.__setitem__)
    acc = [0] * 6
    for i in prog:
        _row(st, i, acc)
    return arena, amp


def scheduled(ins, task_first, level_first, loads, amp_planes, cur_slots, planes, amps, reverse=True):
    arena = [hash(("init", p)) for p in range(planes)]
    amp = [hash(("amp", q)) for q in range(amps)]
    slots = [None] * max(1, cur_slots)
    aslots = [amp[int(p)] for p in amp_planes]
    for j in range(0, len(loads), 3):
        plane, slot, n = (int(v) for v in loads[j:j + 3])
        for k in range(n):
            slots[slot + k] = arena[plane + k]

    def get(sl):
        v = slots[sl]
        assert v is not None, f"slot {sl} read before any write"
        return v

    def put(sl, v):
        slots[sl] = v

    def wb(plane, vals):
        for k, v in enumerate(vals):
            arena[plane + k] = v

    st = _Store(get, put, aslots.__getitem__, aslots.__setitem__)
    for lv in range(len(level_first) - 1):
        tasks = list(range(int(level_first[lv]), int(level_first[lv + 1])))
        if reverse:
            tasks.reverse()
        for t in tasks:
            acc = [0] * 6
            for n in range(int(task_first[t]), int(task_first[t + 1])):
                # the kernel runs sources at level 0 only, and only sources there
                assert (_head(ins[n])[0] == K_SOURCE) == (lv == 0), f"level {lv}: instruction kind {_head(ins[n])[0]}"
                _row(st, ins[n], acc, wb)
    for slot, p in enumerate(amp_planes):
        amp[int(p)] = aslots[slot]
    return arena, amp


def export_terms(words, width, planes, amps, forms, scales, factors, offsets, red_planes):
    """The schedule in reduction-term mode: (applied, ins, task_first, level_first, terms, cur_slots)."""
    keep, a = _args(words, width, planes, amps, forms, scales, factors)
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    rp = np.ascontiguousarray(red_planes, dtype=np.uint32)
    outputs = len(off) - 1
    sizes = np.zeros(8, dtype=np.uint32)
    assert lib().schedule_export_terms(*a, off.ctypes.data, rp.ctypes.data, outputs, sizes.ctypes.data,
                                       None, None, None) == 0
    ins = np.zeros(8 * int(sizes[0]) + 8, dtype=np.uint32)
    tf = np.zeros(int(sizes[1]) + 1, dtype=np.uint32)
    lf = np.zeros(int(sizes[2]) + 1, dtype=np.uint32)
    assert lib().schedule_export_terms(*a, off.ctypes.data, rp.ctypes.data, outputs, sizes.ctypes.data,
                                       ins.ctypes.data, tf.ctypes.data, lf.ctypes.data) == 0
    return (bool(sizes[3]), ins[: 8 * int(sizes[0])].reshape(-1, 8), tf[: int(sizes[1])], lf[: int(sizes[2])],
            int(sizes[4]), int(sizes[5]))


def reference_terms(prog, planes, amps, red_planes):
    """The reduction's terms when every amplitude starts at zero: term k from amplitude red_planes[k]."""
    arena = [hash(("init", p)) for p in range(planes)]
    amp = [ZERO] * amps
    st = _Store(arena.__getitem__, arena.__setitem__, amp.__getitem__, amp.__setitem__)
    acc = [0] * 6
    for i in prog:
        _row(st, i, acc)
    return [hash(("term", amp[int(q)])) for q in red_planes]


def scheduled_terms(ins, task_first, level_first, cur_slots, terms, planes, reverse=True):
    """The terms as the term-mode schedule makes them (no live-in loads: batch plans have none)."""
    slots = [None] * max(1, cur_slots)
    out = [hash(("term", ZERO))] * terms

    def get(sl):
        v = slots[sl]
        assert v is not None, f"slot {sl} read before any write"
        return v

    def put(sl, v):
        slots[sl] = v

    def term_put(t, v):
        out[t] = hash(("term", v))

    def no_amp(*_):
        raise AssertionError("a term-mode schedule touched an amplitude slot")

    st = _Store(get, put, no_amp, no_amp, term_put)
    for lv in range(len(level_first) - 1):
        tasks = list(range(int(level_first[lv]), int(level_first[lv + 1])))
        if reverse:
            tasks.reverse()
        for t in tasks:
            acc = [0] * 6
            for n in range(int(task_first[t]), int(task_first[t + 1])):
                _row(st, ins[n], acc)
    return out
