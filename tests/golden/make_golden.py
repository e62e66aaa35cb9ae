"""Generate the golden fixtures of the parity tests.

For each case: the partition (perm) from the host partitioner and the
oracle's AMLS output (theta, p, kept counts) with dense local eigensolves
(silMode = -1, the semantics the GPU path implements).  The oracle itself is
pinned by the reference's closed-form known answers (tests/test_oracle.py).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from amls_b200 import cases  # noqa: E402
from oracle import amls_ref as R  # noqa: E402
from tests.helpers import partition  # noqa: E402

CASES = {
    "hex8_5x5x5": dict(pencil=["hex", 5, 5, 5, 1, 1], nev=20, nLevels=3, leafSize=100),
    "hex27_3x3x3": dict(pencil=["hex", 3, 3, 3, 2, 4], nev=15, nLevels=3, leafSize=120),
    "grid_30x30": dict(pencil=["grid", 30, 30], nev=20, nLevels=3, leafSize=120),
    "path_500": dict(pencil=["path", 500, 1], nev=15, nLevels=3, leafSize=70),
}


def pencil(spec):
    if spec[0] == "hex":
        return cases.hex_pencil(*spec[1:4], spec[4], seed=spec[5])
    if spec[0] == "grid":
        return cases.grid_graph_2d(spec[1], spec[2])
    return cases.path_graph(spec[1], bool(spec[2]))


def main():
    for name, m in CASES.items():
        p = pencil(m["pencil"])
        perm, tree = partition(p, m["nLevels"], m["leafSize"])
        s = R.amls_solve_ref(p.K, p.M, tree, R.OptionsRef(silMode=-1, nev=m["nev"],
                                                           nLevels=m["nLevels"],
                                                           leafSize=m["leafSize"]))
        np.savez(os.path.join(HERE, f"{name}.npz"), perm=perm, theta=s.theta, p=s.p,
                 k=np.array(s.k), lambda_cut=s.lambda_cut)
        print(name, p.n, "p", s.p, "theta[:3]", s.theta[:3])
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(CASES, f, indent=1)


if __name__ == "__main__":
    main()
