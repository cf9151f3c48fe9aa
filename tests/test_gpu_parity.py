"""Parity of the B200 runner with the CPU oracle and with the reference runner, through the C ABI.

Every scenario (tests/scenarios.py) runs in a fresh process per kernel kind (tests/gpu_worker.py).
The bar is bit-for-bit equality for every kernel kind: the f64 kind against the oracle's f64
restatement and the reference runner's f64 kernel; df64, mixed and mixed64 against the oracle's
restatement of those kernels and the reference's. The reference runner (oracle/_ref, built from
the reference's own sources) is used when it was built.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import scenarios as S
from oracle import oracle as O
from pacuda_b200 import abi, phase_space, processes

ROOT = S.ROOT
LIB = os.path.join(ROOT, "pacuda_b200", "librecurrence.so")
REF = os.path.join(ROOT, "oracle", "_ref", "librecurrence.so")
KINDS = ["f64", "df64", "mixed", "mixed64"]
_cache = {}
_dir = []


def _tmp():
    """A private temporary folder for the workers' outputs (removed at exit)."""
    if not _dir:
        import atexit
        import shutil
        import tempfile

        _dir.append(tempfile.mkdtemp(prefix="pacuda_parity_"))
        atexit.register(shutil.rmtree, _dir[0], True)
    return _dir[0]


def worker(lib, kind, nosort=False, executor=None, lanes=0):
    key = (lib, kind, nosort, executor, lanes)
    if key not in _cache:
        tag = f"{os.path.basename(os.path.dirname(lib))}_{kind}{'_nosort' if nosort else ''}{'_' + executor if executor else ''}" \
            f"{f'_lanes{lanes}' if lanes else ''}"
        out = os.path.join(_tmp(), f"parity_{tag}.npz")
        cmd = [sys.executable, os.path.join(ROOT, "tests", "gpu_worker.py"), lib, kind, out] + (["nosort"] if nosort else []) \
            + ([executor] if executor else []) + ([f"lanes={lanes}"] if lanes else [])
        subprocess.run(cmd, check=True, timeout=600)
        _cache[key] = dict(np.load(out))
    return _cache[key]


def oracle_results(kind):
    k = abi.KERNELS[kind]
    res = {}
    for seed in S.FUZZ_SEEDS:
        a = S.fuzz_args(seed)
        st = O.run(a, kernel=k)
        res[f"fuzz{seed}_status"] = st
        if st == 0:
            res[f"fuzz{seed}_c"] = np.stack([a.cre, a.cim])
            res[f"fuzz{seed}_a"] = np.stack([a.are, a.aim])
    for name in S.PHYSICS:
        amps, outs = O.evaluate(processes.template(name), S.physics_points(name), kernel=k)
        res[f"{name}_amps"] = amps
        res[f"{name}_out"] = outs
    t = processes.template("gg>ggg")
    p = S.physics_points("gg>ggg")
    n = p.shape[0]
    args = t.call(phase_space.source_major(p), n)
    assert O.run(args, kernel=k) == 0
    out = np.linspace(0.5, 1.5, n * t.outputs)
    rr, hold = abi.reduce_resolved_args(t.planes, t.weights, t.offsets, out, n, 1, t.outputs, 0)
    assert O.reduce_resolved(rr, args.are, args.aim, n) == 0
    res["resolved_acc"] = out
    single = np.linspace(-1.0, 1.0, n)
    rs, hold = abi.reduce_args(t.planes[:50], t.weights[:50], single, n)
    assert O.reduce(rs, args.are, args.aim, n) == 0
    res["reduce"] = single
    total, chosen = np.zeros(n), np.zeros(n, dtype=np.uint32)
    random = (np.arange(n) * 0.6180339887498949) % 1.0
    scale = np.where(np.arange(n) % 3 == 0, 1.0 + 0.001 * np.arange(n), 1.0)
    hel = np.arange(t.outputs, dtype=np.uint32) * 3 + 1
    rsa, hold = abi.reduce_sample_args(t.planes, t.weights, t.offsets, hel, n, random, scale, 1.0, 1536.0, total, chosen)
    assert O.reduce_sample(rsa, args.are, args.aim, n) == 0
    res["sample_total"], res["sample_chosen"] = total, chosen
    codes, masses, moms = S.source_cases()
    res["sources"] = O.sources(codes, masses, moms)
    return res


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "c":
        a, b = a.view(np.float64), b.view(np.float64)
    if a.dtype.kind == "f":
        # equal bits, or NaN on both sides (x86 and the GPU write different NaN payloads)
        return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))
    return np.array_equal(a, b)


def compare(got, want, label):
    bad = []
    for key, w in want.items():
        if key not in got:
            bad.append(f"{key}: missing")
            continue
        if not same_bits(got[key], w):
            g = np.asarray(got[key])
            msg = f"{key}: differs"
            if g.dtype.kind in "fc" and g.shape == np.shape(w):
                d = np.abs(g - w)
                scale = max(1e-300, np.abs(w).max())
                msg += f" (max abs {d.max():.3e}, rel to max {d.max() / scale:.3e}, {np.count_nonzero(d)} values)"
            bad.append(msg)
    assert not bad, f"{label}: " + "; ".join(bad[:8])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_runner_matches_oracle_bitwise(kind):
    """The default executor (the on-chip one whenever a plan's points fit)."""
    compare(worker(LIB, kind), oracle_results(kind), f"runner {kind} vs oracle")


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("executor", ["arena", "onchip"])
def test_each_executor_matches_oracle_bitwise(kind, executor):
    compare(worker(LIB, kind, executor=executor), oracle_results(kind), f"runner {kind} ({executor}) vs oracle")


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [8, 96, 512])
def test_configured_lanes_per_point_match_oracle_bitwise(lanes):
    """The C ABI's on-chip runs at 32, 5 and 1 points per block (plans whose points do not fit
    run on the global-arena executor)."""
    compare(worker(LIB, "f64", lanes=lanes), oracle_results("f64"), f"runner f64 ({lanes} lanes) vs oracle")


@pytest.mark.gpu
def test_f64_unsorted_equals_sorted():
    a, b = worker(LIB, "f64"), worker(LIB, "f64", nosort=True)
    compare(b, a, "f64 no_sort vs sort")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference runner not built (make -C oracle ref)")
@pytest.mark.parametrize("kind", KINDS)
def test_runner_matches_reference_runner_bitwise(kind):
    compare(worker(LIB, kind), worker(REF, kind), f"runner {kind} vs reference runner {kind}")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference runner not built (make -C oracle ref)")
def test_oracle_matches_reference_runner_f64():
    """The oracle's pin: its f64 restatement equals the reference runner's f64 kernel."""
    compare(worker(REF, "f64"), oracle_results("f64"), "reference runner f64 vs oracle")


RECTEST = os.path.join(ROOT, "oracle", "_ref", "rectest")


def rectest(lib, *args):
    p = subprocess.run([RECTEST, lib, *args], capture_output=True, text=True, timeout=300)
    return p.returncode, p.stdout, p.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(RECTEST), reason="reference rectest not built (make -C oracle ref)")
@pytest.mark.parametrize("args", [("f64",), ("f64", "nosort"), ("df64",), (), ("mixed",), ("mixed64",)])
def test_reference_rectest_passes_on_this_runner(args):
    """The reference's own runner test (runner/rectest.c, built unmodified) against this library:
    its device reductions equal its host reductions bit for bit, kept amplitudes are not copied
    back; and the amplitudes it prints equal the reference runner's, kernel for kernel."""
    code, out, err = rectest(LIB, *args)
    assert code == 0, err
    if os.path.exists(REF):
        rcode, rout, rerr = rectest(REF, *args)
        assert rcode == 0, rerr
        assert out == rout, "rectest amplitudes differ from the reference runner's"


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(RECTEST), reason="reference rectest not built (make -C oracle ref)")
def test_rectest_variants_agree():
    """tests/runner_variants.sh's bar: f64 sorted == unsorted; df64 within 1e-9, mixed and mixed64
    within 1e-4 of the largest f64 value."""
    outs = {k: rectest(LIB, *k.split())[1] for k in ["f64", "f64 nosort", "df64", "mixed", "mixed64"]}
    assert outs["f64"] == outs["f64 nosort"]
    want = np.array(outs["f64"].split(), dtype=float)
    assert want.size == 3 * 300 * 2 and np.any(want)
    scale = np.abs(want).max()
    for k, tol in [("df64", 1e-9), ("mixed", 1e-4), ("mixed64", 1e-4)]:
        got = np.array(outs[k].split(), dtype=float)
        assert np.abs(got - want).max() / scale <= tol, k
