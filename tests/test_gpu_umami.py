"""The UMAMI library on the GPU: every mode's |M|^2 (helicity sum, a fixed helicity, helicity
sampling, another alpha_s) equals, bit for bit, the reference library's arithmetic applied to the
oracle's helicity values (tests/umami_fixture.py); with the colour and helicity indices, its error
statuses and its parameters."""
import ctypes as C

import numpy as np
import pytest

from tests import umami_fixture as U

COUNT, STRIDE, OFFSET = 700, 1000, 37


@pytest.fixture(scope="module")
def umami(tmp_path_factory):
    from pacuda_b200 import build
    from pacuda_b200.umami import build as ubuild, provider

    build.build()
    d = tmp_path_factory.mktemp("umami")
    hdr = d / "provider_test.h"
    hdr.write_text(provider.header(U.SPEC))
    lib = C.CDLL(ubuild.build(str(hdr), str(d / "libumami_test.so")))
    lib.umami_initialize.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
    lib.umami_matrix_element.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p)]
    lib.umami_set_parameter.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double]
    lib.umami_get_parameter.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.umami_free.argtypes = [C.c_void_p]
    h = C.c_void_p()
    assert lib.umami_initialize(C.byref(h), U.make_artifact(str(d / "artifact")).encode()) == 0
    yield lib, h
    assert lib.umami_free(h) == 0


def call(umami, ins, outs, count=COUNT, stride=STRIDE, offset=OFFSET):
    lib, h = umami
    ik = (C.c_int * len(ins))(*[k for k, _ in ins])
    ip = (C.c_void_p * len(ins))(*[a.ctypes.data for _, a in ins])
    ok = (C.c_int * len(outs))(*[k for k, _ in outs])
    op = (C.c_void_p * len(outs))(*[a.ctypes.data for _, a in outs])
    return lib.umami_matrix_element(h, count, stride, offset, len(ins), ik, ip, len(outs), ok, op)


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["sum", "helicity", "sample", "sample alpha_s 0.13"])
def test_every_mode_matches_the_references_arithmetic_bitwise(umami, mode):
    from oracle import oracle as O

    sample = mode.startswith("sample")
    m, p, channel, flavour = U.events(COUNT, STRIDE, OFFSET, single=sample)
    rng = np.random.default_rng(5)
    alpha = np.full(STRIDE, 0.13 if "0.13" in mode else 0.118)
    random = rng.random(STRIDE)
    helicity = rng.integers(0, 32, STRIDE).astype(np.int32)
    me, col, hel = np.full(STRIDE, -1.0), np.full(STRIDE, -1, np.int32), np.full(STRIDE, -1, np.int32)
    ins = [(0, m), (1, alpha), (2, flavour), (8, channel)]
    outs = [(0, me), (2, col)]
    if sample:
        ins.append((4, random))
        outs.append((3, hel))
    elif mode == "helicity":
        ins.append((6, helicity))
    want_me, want_col, want_hel = U.expected(p, channel, flavour, OFFSET, "sample" if sample else mode, O,
                                             alpha=alpha, random=random, helicity=helicity)
    for repeat in range(2):  # the second call reuses the first's batch
        me[:] = -1.0
        assert call(umami, ins, outs) == 0
        got = me[OFFSET:OFFSET + COUNT]
        assert same_bits(got, want_me), (repeat, np.abs(got / want_me - 1).max())
        assert np.array_equal(col[OFFSET:OFFSET + COUNT], want_col)
        if sample:
            assert np.array_equal(hel[OFFSET:OFFSET + COUNT], want_hel)
        assert np.all(me[:OFFSET] == -1.0) and np.all(me[OFFSET + COUNT:] == -1.0)


@pytest.mark.gpu
def test_a_call_with_other_groups_and_fewer_events(umami):
    from oracle import oracle as O

    m, p, channel, flavour = U.events(COUNT, STRIDE, OFFSET)
    channel[:] = 0
    flavour[:] = 0
    me = np.zeros(STRIDE)
    n = 50
    assert call(umami, [(0, m), (2, flavour), (8, channel)], [(0, me)], count=n) == 0
    want, _, _ = U.expected(p[:n], channel, flavour, OFFSET, "sum", O)
    assert same_bits(me[OFFSET:OFFSET + n], want)


@pytest.mark.gpu
def test_statuses(umami):
    m, p, channel, flavour = U.events(COUNT, STRIDE, OFFSET)
    me, hel = np.zeros(STRIDE), np.zeros(STRIDE, np.int32)
    base = [(0, m), (2, flavour), (8, channel)]
    assert call(umami, base + [(3, m)], [(0, me)]) == 2                      # a key it does not take
    assert call(umami, [(2, flavour), (8, channel)], [(0, me)]) == 5         # no momenta
    bad = np.full(STRIDE, 1.0)
    assert call(umami, base + [(4, bad)], [(0, me)]) == 1                   # random number outside [0, 1)
    two = flavour.copy()
    two[OFFSET:OFFSET + COUNT] = np.where(channel[OFFSET:OFFSET + COUNT] == 1, 2, 0)
    assert call(umami, [(0, m), (2, two), (8, channel)], [(0, me), (3, hel)]) == 3  # sampling over two contributions
    nan = m.copy()
    nan[OFFSET + STRIDE * 3] = np.nan
    assert call(umami, [(0, nan), (2, flavour), (8, channel)], [(0, me)]) == 1
    assert call(umami, base, [(0, me)], count=0) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("first", ["random", "sampling"])
def test_the_first_failing_event_decides_the_status(umami, first):
    """Of two failing events far apart in one chunk, the earlier one's status is the call's, as
    the reference's checks in event order give it (a random number outside [0, 1): 1; sampling
    over two contributions: 3)."""
    count = stride = 100000
    m, p, channel, flavour = U.events(count, stride, 0, seed=5, single=True)
    random = np.random.default_rng(3).random(stride)
    me, hel = np.zeros(stride), np.zeros(stride, np.int32)
    early, late = 20000, 80000
    bad_random, two = (early, late) if first == "random" else (late, early)
    random[bad_random] = 1.0
    channel[two], flavour[two] = 1, 2
    status = call(umami, [(0, m), (2, flavour), (8, channel), (4, random)], [(0, me), (3, hel)], count=count,
                  stride=stride, offset=0)
    assert status == (1 if first == "random" else 3)


@pytest.mark.gpu
def test_parameters(umami):
    from oracle import oracle as O

    lib, h = umami
    re, im = C.c_double(), C.c_double()
    assert lib.umami_get_parameter(h, b"aS", C.byref(re), C.byref(im)) == 0 and re.value == 0.118
    assert lib.umami_get_parameter(h, b"MT", C.byref(re), C.byref(im)) == 0 and re.value == 173.0
    assert lib.umami_set_parameter(h, b"MT", 173.0, 0.0) != 0   # not mutable
    assert lib.umami_set_parameter(h, b"ymt", 175.0, 0.0) != 0  # mutable, but the file holds 173
    assert lib.umami_set_parameter(h, b"ymt", 173.0, 0.0) == 0  # its value at conversion is accepted
    assert lib.umami_set_parameter(h, b"nope", 1.0, 0.0) != 0
    assert lib.umami_set_parameter(h, b"aS", 0.13, 0.0) == 0
    try:
        assert lib.umami_get_parameter(h, b"aS", C.byref(re), C.byref(im)) == 0 and re.value == 0.13
        m, p, channel, flavour = U.events(COUNT, STRIDE, OFFSET)
        me = np.zeros(STRIDE)
        assert call(umami, [(0, m), (2, flavour), (8, channel)], [(0, me)]) == 0
        want, _, _ = U.expected(p, channel, flavour, OFFSET, "sum", O, alpha=np.full(STRIDE, 0.13))
        assert same_bits(me[OFFSET:OFFSET + COUNT], want)
    finally:
        assert lib.umami_set_parameter(h, b"aS", 0.118, 0.0) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("mode,count", [("sum", 3 * 65536 + 123), ("sample", 3 * 65536 + 123),
                                        ("sum", 6 * 65536 + 5)])
def test_a_call_of_several_chunks(umami, mode, count):
    """A call of more than 2^17 events is evaluated in chunks whose host and device work overlap
    (three equal chunks, or the five growing chunks of a full call)."""
    from oracle import oracle as O

    stride, offset = count + 77, 11
    m, p, channel, flavour = U.events(count, stride, offset, seed=23, single=mode == "sample")
    random = np.random.default_rng(9).random(stride)
    me, hel = np.full(stride, -1.0), np.full(stride, -1, np.int32)
    ins = [(0, m), (2, flavour), (8, channel)]
    outs = [(0, me)]
    if mode == "sample":
        ins.append((4, random))
        outs.append((3, hel))
    assert call(umami, ins, outs, count=count, stride=stride, offset=offset) == 0
    want_me, _, want_hel = U.expected(p, channel, flavour, offset, mode, O, random=random)
    assert same_bits(me[offset:offset + count], want_me)
    if mode == "sample":
        assert np.array_equal(hel[offset:offset + count], want_hel)



@pytest.mark.gpu
def test_six_gluon_subprocess_sums_its_colour_parts(tmp_path):
    """A gg>gggg subprocess whose one flavour lists the process's three plan parts as three
    colour contributions: the helicity sum of |M|^2 is their sum, as the reference library adds a
    flavour's contributions, bit for bit against the oracle's values."""
    from oracle import oracle as O
    from pacuda_b200 import build, pacuda_file, phase_space, processes
    from pacuda_b200.umami import build as ubuild, provider

    build.build()
    parts = processes.parts("gg>gggg")
    spec = {"particles": 6, "masses": [0.0] * 6, "colors": 1,
            "processes": [{"key": "gg>gggg", "helicities": 64, "parameters": [("aS", 0.118, 0.0, False, True)]}],
            "channels": [[[{"process": 0, "colour": f"lc{k}", "permutation": list(range(6)), "factor": 1.0}
                           for k in range(len(parts))]]],
            "has_alpha_s": True, "has_color_flow": False}
    hdr = tmp_path / "provider_6g.h"
    hdr.write_text(provider.header(spec))
    lib = C.CDLL(ubuild.build(str(hdr), str(tmp_path / "libumami_6g.so")))
    lib.umami_initialize.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
    lib.umami_matrix_element.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p)]
    lib.umami_free.argtypes = [C.c_void_p]
    art = tmp_path / "artifact6"
    art.mkdir()
    pacuda_file.write(pacuda_file.from_processes(["gg>gggg"], reference_points=0), str(art) + ".pacuda")
    h = C.c_void_p()
    assert lib.umami_initialize(C.byref(h), str(art).encode()) == 0
    n = 300
    p = phase_space.sample(6, n, 17, ecm=13000.0)
    m = np.ascontiguousarray(p.transpose(2, 1, 0).reshape(24, n))  # [6 k + leg][event]
    me = np.zeros(n)
    ik, ip = (C.c_int * 1)(0), (C.c_void_p * 1)(m.ctypes.data)
    ok, op = (C.c_int * 1)(0), (C.c_void_p * 1)(me.ctypes.data)
    try:
        assert lib.umami_matrix_element(h, n, n, 0, 1, ik, ip, 1, ok, op) == 0
    finally:
        lib.umami_free(h)
    num, den = parts[0].meta["group_factor"]
    total = np.zeros(n)
    for t in parts:
        _, out = O.evaluate(t, p, kernel=1)
        live = np.asarray(t.offsets[1:]) > np.asarray(t.offsets[:-1])
        v = out * float(num) / float(den)
        v[:, ~live] = 0.0
        value = np.zeros(n)
        for hel in range(v.shape[1]):
            value = value + v[:, hel]
        total = total + 1.0 * value
    assert same_bits(me, total)
