"""Runs the shared scenarios on a runner library in this process and saves what came back.

usage: python tests/gpu_worker.py LIB KERNEL OUT.npz [nosort] [arena|onchip] [lanes=N]

One process per kernel kind, since a runner takes its configuration once, before its first run.
LIB is this package's librecurrence.so or the reference runner built from its sources.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from tests import scenarios as S  # noqa: E402
from pacuda_b200 import abi, phase_space, processes  # noqa: E402
from pacuda_b200.runner import Runner  # noqa: E402


def main():
    lib, kernel, path = sys.argv[1], sys.argv[2], sys.argv[3]
    no_sort = "nosort" in sys.argv[4:]
    executor = "arena" if "arena" in sys.argv[4:] else "onchip" if "onchip" in sys.argv[4:] else None
    lanes = [int(a[6:]) for a in sys.argv[4:] if a.startswith("lanes=")]
    r = Runner(lib)
    if lanes:
        assert r.configure(kernel, no_sort=no_sort, executor=executor, lanes_per_point=lanes[0]) == 0
    else:
        assert r.configure(kernel, no_sort=no_sort, executor=executor) == 0
    res = {}
    for seed in S.FUZZ_SEEDS:
        a = S.fuzz_args(seed)
        st = r.run(a)
        res[f"fuzz{seed}_status"] = np.array(st)
        if st == 0:
            res[f"fuzz{seed}_c"] = np.stack([a.cre, a.cim])
            res[f"fuzz{seed}_a"] = np.stack([a.are, a.aim])
    for name in S.PHYSICS:
        t = processes.template(name)
        p = S.physics_points(name)
        amps, outs = r.evaluate(t, p)
        res[f"{name}_amps"] = amps
        res[f"{name}_out"] = outs
    # the three reductions of a kept run (gg>ggg)
    t = processes.template("gg>ggg")
    p = S.physics_points("gg>ggg")
    n = p.shape[0]
    ext = phase_space.source_major(p)
    keep = t.call(ext, n)
    assert r.run(keep) == 0
    out = np.linspace(0.5, 1.5, n * t.outputs)
    rr, hold = abi.reduce_resolved_args(t.planes, t.weights, t.offsets, out, n, 1, t.outputs, 0)
    assert r.reduce_resolved(rr) == 0
    res["resolved_acc"] = out.copy()
    assert r.run(keep) == 0
    single = np.linspace(-1.0, 1.0, n)
    rs, hold = abi.reduce_args(t.planes[:50], t.weights[:50], single, n)
    assert r.reduce(rs) == 0
    res["reduce"] = single.copy()
    assert r.run(keep) == 0
    total = np.zeros(n)
    chosen = np.zeros(n, dtype=np.uint32)
    random = (np.arange(n) * 0.6180339887498949) % 1.0
    scale = np.where(np.arange(n) % 3 == 0, 1.0 + 0.001 * np.arange(n), 1.0)
    hel = np.arange(t.outputs, dtype=np.uint32) * 3 + 1
    rsa, hold = abi.reduce_sample_args(t.planes, t.weights, t.offsets, hel, n, random, scale, 1.0, 1536.0, total, chosen)
    assert r.reduce_sample(rsa) == 0
    res["sample_total"] = total
    res["sample_chosen"] = chosen
    # sources of every family through the test entry point
    codes, masses, moms = S.source_cases()
    res["sources"] = r.test_sources(codes, masses, moms)
    np.savez(path, **res)


if __name__ == "__main__":
    main()
