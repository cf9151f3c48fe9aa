"""Evaluates the small plain-method configuration through one runner library in this process and
saves what came back: g g -> g g g, leading colour (12 orderings x 32 helicities), 4096 seeded
RAMBO points at sqrt(s) = 1 TeV with pT > 20 GeV, |eta| < 5, Delta R > 0.4, in f64.

usage: python tests/c0_worker.py LIB OUT.npz [batch]

Through the library's C ABI: a run with its amplitudes downloaded, then a kept run reduced on the
device by reduce_resolved. With `batch` (this package's library only): the same points through
the batched device API (pacuda_b200_batch_run) as well.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from pacuda_b200 import phase_space, processes  # noqa: E402
from pacuda_b200.runner import Runner  # noqa: E402

POINTS, ECM, SEED = 4096, 1000.0, 4096


def points():
    return phase_space.sample(5, POINTS, SEED, ecm=ECM)


def main():
    lib, path = sys.argv[1], sys.argv[2]
    t = processes.template("gg>ggg")
    p = points()
    r = Runner(lib)
    assert r.configure("f64") == 0
    amps, outs = r.evaluate(t, p)
    res = {"abi_amps": amps, "abi_out": outs}
    if "batch" in sys.argv[3:]:
        import torch

        from pacuda_b200 import batch as B

        plan = B.Plan(t, "f64")
        ext = torch.tensor(phase_space.source_major(p), dtype=torch.float64, device="cuda")
        out = torch.empty(POINTS * t.outputs, dtype=torch.float64, device="cuda")
        b = B.Batch([plan], [ext], [out])
        b.tune()
        b.run()
        torch.cuda.synchronize()
        res["batch_out"] = out.cpu().numpy().reshape(POINTS, t.outputs)
    np.savez(path, **res)


if __name__ == "__main__":
    main()
