"""Golden vectors for the full-size workload (27-node hex, 14^3 elements,
70,644 DOF, nev 500, nLevels 8, eta 2), generated on the CPU:

  c5_oracle.npz  the oracle's AMLS output (theta, p, p of pass A, perm)
                 with the reference's default local eigensolver choice
                 (silMode 0: the two leaves of 441 DOF whose K_ii has fewer
                 than 0.15 n^2 nonzero values take the shift-invert branch);
  c5_exact.npz   the 520 smallest exact eigenvalues by shift-invert Lanczos
                 (scipy ARPACK, sigma = 0, tol 1e-13), standing in for the
                 reference's Spectra SymGEigsShiftSolver path
                 (src/reference/reference_solver.cpp:39-94);
  c5_tree.npz    the separator tree of the partition (parent, role, left,
                 right, node index lists), so that the CPU baseline runs the
                 oracle on the same tree without calling the partitioner.

Run from the repository root (takes several minutes):
  python tests/golden/make_c5_golden.py [oracle|exact|tree|both]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from amls_b200 import cases  # noqa: E402
from oracle import amls_ref as R  # noqa: E402
from amls_b200.solver import recursive_bisection  # noqa: E402
from tests.helpers import partition  # noqa: E402


def main(which):
    p = cases.config_pencil("C5", seed=0)
    if which in ("oracle", "both"):
        perm, tree = partition(p, 8, 500)
        t = time.time()
        s = R.amls_solve_ref(p.K, p.M, tree, R.OptionsRef(nev=500, nLevels=8, silMode=0,
                                                           recoverVectors=False))
        print("oracle", time.time() - t, "p", s.p, "pA", s.p_passA, flush=True)
        np.savez(os.path.join(HERE, "c5_oracle.npz"), theta=s.theta, p=s.p, p_passA=s.p_passA,
                 perm=perm, lambda_cut=s.lambda_cut)
    if which in ("tree", "both"):
        perm, t = recursive_bisection(p.K, p.M, 8, 500)
        np.savez_compressed(os.path.join(HERE, "c5_tree.npz"), perm=perm.astype(np.int32),
                            parent=t["parent"].astype(np.int32), role=t["role"].astype(np.int32),
                            left=t["left"].astype(np.int32), right=t["right"].astype(np.int32),
                            idx_ptr=t["idx_ptr"].astype(np.int32), idx=t["idx"].astype(np.int32))
    if which in ("exact", "both"):
        import scipy.sparse as sp
        import scipy.sparse.linalg as spla
        t = time.time()
        w = spla.eigsh(sp.csc_matrix(p.K), k=520, M=sp.csc_matrix(p.M), sigma=0.0, which="LM",
                       ncv=1200, tol=1e-13, return_eigenvectors=False)
        w = np.sort(w)
        print("exact", time.time() - t, w[:3], w[-3:], flush=True)
        np.savez(os.path.join(HERE, "c5_exact.npz"), theta=w)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "both")
