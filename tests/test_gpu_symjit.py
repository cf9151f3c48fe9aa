"""Symjit rows (ops 13/14) in a runner built without generated symjit kernels: the run is refused
with DEVICE_ERROR (3) as the reference refuses it (runner/recurrence_runner.cu:1141-1145), the
capability bit 2 is clear (:1785-1788) and symjit_kernel answers -1, for this library and the
reference runner built from its sources alike; the runner keeps working after the refusal."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from pacuda_b200.runner import Runner
from tests.test_gpu_parity import LIB, REF, ROOT


def run_worker(lib):
    with tempfile.TemporaryDirectory(prefix="pacuda_symjit_") as d:
        out = os.path.join(d, "s.npz")
        subprocess.run([sys.executable, os.path.join(ROOT, "tests", "symjit_worker.py"), lib, out], check=True,
                       timeout=300)
        return {k: int(v) for k, v in np.load(out).items()}


def test_capabilities_without_symjit_kernels():
    """Host-only entry points (no device work): sources and device forms, no symjit kernels."""
    r = Runner(LIB)
    assert r.capabilities() == 1 | 2
    assert r.symjit_kernel("0" * 64) == -1 and r.symjit_kernel("") == -1


@pytest.mark.gpu
def test_symjit_rows_are_refused():
    got = run_worker(LIB)
    assert got == {"status": 3, "after": 0, "caps": 3, "kernel": -1}


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference runner not built (make -C oracle ref)")
def test_symjit_refusal_matches_the_reference_runner():
    assert run_worker(LIB) == run_worker(REF)
