"""The small plain-method configuration at its full size, bit for bit: g g -> g g g, leading
colour, all 12 orderings and 32 helicities, 4096 RAMBO points at sqrt(s) = 1 TeV with pT > 20 GeV,
|eta| < 5 and Delta R > 0.4, in f64. Through the C ABI (a run with downloaded amplitudes, a kept
run reduced by reduce_resolved) and through the batched device API, against the oracle and
against the reference runner built from its own sources (oracle/_ref)."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from pacuda_b200 import abi, processes
from tests import c0_worker as W
from tests.test_gpu_parity import LIB, REF, ROOT, same_bits

_res = {}


def run_worker(lib, *extra):
    key = (lib,) + extra
    if key not in _res:
        with tempfile.TemporaryDirectory(prefix="pacuda_c0_") as d:
            out = os.path.join(d, "c0.npz")
            subprocess.run([sys.executable, os.path.join(ROOT, "tests", "c0_worker.py"), lib, out, *extra], check=True,
                           timeout=600)
            _res[key] = dict(np.load(out))
    return _res[key]


def oracle_c0():
    if "oracle" not in _res:
        amps, outs = O.evaluate(processes.template("gg>ggg"), W.points(), kernel=abi.KERNEL_F64)
        _res["oracle"] = {"amps": amps, "out": outs}
    return _res["oracle"]


def test_c0_points_are_the_configuration():
    """CPU check of the inputs: 4096 points, massless, momentum conserved, every cut passed."""
    p = W.points()
    assert p.shape == (4096, 5, 4)
    assert np.allclose(p[:, :, 0] ** 2 - (p[:, :, 1:] ** 2).sum(axis=2), 0.0, atol=1e-6)
    assert np.allclose(p[:, :2].sum(axis=1), p[:, 2:].sum(axis=1), atol=1e-9)
    assert p[:, :2, 0].sum(axis=1) == pytest.approx(np.full(4096, 1000.0))
    from pacuda_b200 import phase_space

    assert phase_space.passes_cuts(p).all()


@pytest.mark.gpu
def test_c0_abi_and_batch_equal_the_oracle_bitwise():
    got = run_worker(LIB, "batch")
    want = oracle_c0()
    assert same_bits(got["abi_amps"], want["amps"])
    assert same_bits(got["abi_out"], want["out"])
    assert same_bits(got["batch_out"], want["out"])
    assert np.all(want["out"].sum(axis=1) > 0)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference runner not built (make -C oracle ref)")
def test_c0_equals_the_reference_runner_bitwise():
    got, ref = run_worker(LIB, "batch"), run_worker(REF)
    assert same_bits(got["abi_amps"], ref["abi_amps"])
    assert same_bits(got["abi_out"], ref["abi_out"])
    assert same_bits(got["batch_out"], ref["abi_out"])
