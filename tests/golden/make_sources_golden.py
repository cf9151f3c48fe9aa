"""Generates tests/golden/sources_legend.npz: external wavefunctions from the reference's own
legend of them.

The reference's tests/check_sources.py restates convert/CONVENTIONS.md's source legend in Python
(`w(name, k, h, ch, m)`) and compares a runner's `pacman_recurrence_v1_test_sources` with it.
This script loads only that file's function definitions (by AST, from the mounted reference;
nothing of it is copied here), evaluates them on seeded cases of every family, orientation,
helicity and chirality, both energy signs and the pT = 0 and p = 0 edge cases, and stores the
cases and the legend's values. The oracle must agree with them to 1e-13 relative, the
reference's own bar (check_sources.py:105).

usage: python tests/golden/make_sources_golden.py [reference source tree]
"""
import ast
import math
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's source tree: the first argument, $PACUDA_REFERENCE, else a checkout named
# `reference` beside this repository
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
    "PACUDA_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))


def legend():
    src = open(os.path.join(REF, "tests", "check_sources.py")).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef)]
    keep += [n for n in tree.body if isinstance(n, ast.Assign) and any(
        isinstance(t, ast.Name) and t.id == "sq2" for t in n.targets)]
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {"math": math}
    exec(compile(mod, "check_sources_legend", "exec"), ns)
    return ns["w"]


def main():
    w = legend()
    rng = random.Random(20261203)
    families = {"scalar": (0, 0), "weyl particle": (1, 0), "weyl antiparticle": (1, 1), "dirac particle": (2, 0),
                "dirac antiparticle": (2, 1), "vector (massless)": (3, 0), "vector (massive)": (3, 0)}
    codes, masses, moms, values, names = [], [], [], [], []
    for name, (fam, ori) in families.items():
        for _ in range(200):
            if name.startswith("dirac"):
                m = rng.choice([0.0, 4.7, 91.188, 173.0])
            elif name == "vector (massive)":
                m = rng.choice([80.4, 91.188])
            else:
                m = 0.0
            kind = rng.random()
            if kind < 0.15:
                p3 = [0.0, 0.0, rng.choice([-1, 1]) * rng.uniform(1, 500)]
            elif kind < 0.2:
                p3 = [0.0, 0.0, 0.0]
            else:
                p3 = [rng.uniform(-500, 500) for _ in range(3)]
            e = math.sqrt(sum(x * x for x in p3) + m * m)
            if e == 0:
                continue
            sgn = rng.choice([1, -1])
            k = [sgn * e] + [sgn * x for x in p3]
            hs = [0] if fam == 0 else ([-1, 0, 1] if name == "vector (massive)" else [-1, 1])
            h = rng.choice(hs)
            ch = rng.choice([-1, 1]) if fam == 1 else 0
            code = fam | ori << 3 | (h + 2) << 5 | (ch + 1) << 8
            got = [complex(x) for x in w(name, k, h, ch, m)] + [0j] * 4
            codes.append(code)
            masses.append(m)
            moms.append(k)
            values.append(got[:4])
            names.append(name)
    np.savez(os.path.join(HERE, "sources_legend.npz"), codes=np.array(codes, dtype=np.uint32), masses=np.array(masses),
             momenta=np.array(moms), values=np.array(values), names=np.array(names))
    print(f"{len(codes)} cases")


if __name__ == "__main__":
    main()
