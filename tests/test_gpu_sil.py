"""Shift-invert Lanczos (SIL) nodes on the GPU against the oracle run with
the same local eigensolver choice (the reference's EigenpairSolver::silMode,
src/amls/eigenpair_solver.hpp:28-29, 68-82; the Lanczos of
src/amls/shift_invert_lanczos.hpp:32-203 with its ncv schedule, start vector
and selection).  Tolerance: theta within 1e-10 relative of the oracle's, same
reduced size p.

The automatic case is the reference's own regression case (grid 64 x 64,
nev 50, eta 2, nLevels 4, leafSize 1000; tests/regression/test_regression.cpp:
37-52): its four leaves of ~990 DOF have nnz/n^2 ~ 0.005, so the reference's
default solve takes the SIL branch there, and the result is within the
reference's 4 % of the closed-form spectrum.
"""
import numpy as np
import pytest

from amls_b200 import AmlsOptions, cases
from oracle import amls_ref as R

from .helpers import oracle_solve, rel_err

pytestmark = pytest.mark.gpu


def test_sil_auto_grid64_matches_oracle(solver):
    p = cases.grid_graph_2d(64, 64)
    o = dict(nev=50, nLevels=4, leafSize=1000)
    ref = oracle_solve(p, R.OptionsRef(silMode=0, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(silMode=0, **o))
    assert sol.info["sil_nodes"] == 4 and sol.info["sil_served"] == 4
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10
    exact = cases.grid_graph_2d_spectrum(64, 64)[:50]
    assert rel_err(sol.theta, exact) <= 0.04          # test_regression.cpp:51
    mn = np.einsum("ij,ij->j", sol.Z, p.M @ sol.Z)
    assert np.allclose(mn, 1.0, atol=1e-12)


@pytest.mark.parametrize("case", ["hex8_5", "grid_40", "path_600"])
def test_sil_forced_matches_oracle(solver, case):
    """silMode = 1: every node (separators included) through the Lanczos
    path, index mode in pass A (falling back to dense where k >= 4n/5) and
    interval mode with the ncv doubling in pass B."""
    if case == "hex8_5":
        p = cases.hex_pencil(5, 5, 5, 1, seed=1)
        o = dict(nev=20, nLevels=3, leafSize=100)
    elif case == "grid_40":
        p = cases.grid_graph_2d(40, 40)
        o = dict(nev=30, nLevels=4, leafSize=150)
    else:
        p = cases.path_graph(600, True)
        o = dict(nev=25, nLevels=4, leafSize=60)
    ref = oracle_solve(p, R.OptionsRef(silMode=1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(silMode=1, **o))
    assert sol.info["sil_nodes"] == sol.info["tree_nodes"]
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10


def test_sil_forced_fixed_keep_and_refined(solver):
    """Forced SIL with a fixed count per node, then the FP64 refinement to
    the exact eigenvalues (dense LAPACK)."""
    p = cases.hex_pencil(6, 5, 4, 1, seed=7)
    o = dict(nev=12, nLevels=3, leafSize=80, fixedKeep=6)
    ref = oracle_solve(p, R.OptionsRef(silMode=1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(silMode=1, **o))
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    fine = solver.solve(p.K, p.M, AmlsOptions(silMode=1, refine=3, nev=12, nLevels=3, leafSize=80))
    assert rel_err(fine.theta, wr[:12]) < 1e-8


def test_sil_off_matches_dense_oracle(solver):
    """silMode = -1 keeps every node dense (the round-trip of the knob)."""
    p = cases.grid_graph_2d(64, 64)
    o = dict(nev=50, nLevels=4, leafSize=1000)
    ref = oracle_solve(p, R.OptionsRef(silMode=-1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(silMode=-1, **o))
    assert sol.info["sil_nodes"] == 0
    assert rel_err(sol.theta, ref.theta) < 1e-10
