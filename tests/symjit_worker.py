"""Runs a plan with symjit rows (op 14 binding + op 13 row) through one runner library and saves
its status, capabilities and symjit_kernel answer.

usage: python tests/symjit_worker.py LIB OUT.npz
"""
import dataclasses
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from pacuda_b200 import phase_space, processes  # noqa: E402
from pacuda_b200.runner import Runner  # noqa: E402


def symjit_plan():
    """gg>ggg with a binding (kernel 0, one input, one output pair) and a symjit row after its
    rows: an op 13 row needs a generated kernel, which a runner without symjit kernels refuses."""
    t = processes.template("gg>ggg")
    binding = np.uint64(14 | 0 << 4 | 1 << 20 | 1 << 28)
    data = np.uint64(0 | 0 << 32)  # input code: parent 0, component 0, real part; output component 0
    row = np.uint64(13 | 1 << 4 | 5 << 5)  # init, parent 0 = plane 5 (width P starts at bit 5)
    return dataclasses.replace(t, words=np.concatenate([t.words, [binding, data, row]]).astype(np.uint64))


def main():
    lib, path = sys.argv[1], sys.argv[2]
    r = Runner(lib)
    assert r.configure("f64") == 0
    t = symjit_plan()
    p = phase_space.sample(5, 64, 5)
    status = r.run(t.call(phase_space.source_major(p), 64, words_key=0))
    # the same runner still runs a plan without symjit rows afterwards
    ok = r.run(processes.template("gg>ggg").call(phase_space.source_major(p), 64))
    np.savez(path, status=status, after=ok, caps=r.capabilities(), kernel=r.symjit_kernel("0" * 64))


if __name__ == "__main__":
    main()
