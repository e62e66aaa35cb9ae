"""The C++ restatement of the reference algorithm (oracle/amls_cpu.cpp, the
timed CPU baseline) against the Python restatement (oracle/amls_ref.py) on
the same partition trees: same reduced sizes, eigenvalues within 1e-10, M-
normalised vectors.  CPU only."""
import numpy as np
import pytest

from amls_b200 import cases
from amls_b200.solver import recursive_bisection
from oracle import amls_ref as R
from oracle import cpu
from oracle.tree import Tree


@pytest.mark.parametrize("case", ["hex8_5", "hex27_3", "C1", "fixed_keep"])
def test_cpp_restatement_matches_python_restatement(case):
    fixed = 0
    if case == "hex8_5":
        p, o = cases.hex_pencil(5, 5, 5, 1, seed=1), dict(nev=20, nLevels=3, leafSize=100)
    elif case == "hex27_3":
        p, o = cases.hex_pencil(3, 3, 3, 2, seed=4), dict(nev=15, nLevels=3, leafSize=120)
    elif case == "C1":
        p, o = cases.config_pencil("C1"), dict(nev=20, nLevels=4, leafSize=500)
    else:
        p, o = cases.hex_pencil(6, 5, 4, 1, seed=7), dict(nev=12, nLevels=3, leafSize=80)
        fixed = 6
    _, t = recursive_bisection(p.K, p.M, o["nLevels"], o["leafSize"])
    ref = R.amls_solve_ref(p.K, p.M, Tree.from_arrays(**t), R.OptionsRef(silMode=-1, fixedKeep=fixed, **o))
    th, Z, pp, pa, tm = cpu.solve(p.K, p.M, t, o["nev"], fixed_keep=fixed, threads=4)
    assert pp == ref.p and pa == ref.p_passA
    assert np.max(np.abs(th - ref.theta) / ref.theta) < 1e-10
    mn = np.einsum("ij,ij->j", Z, p.M @ Z)
    assert np.allclose(mn, 1.0, atol=1e-12)
    # same Ritz vectors up to sign
    s = np.sign(np.einsum("ij,ij->j", Z, p.M @ ref.Z))
    assert np.max(np.abs(Z * s - ref.Z)) < 1e-7 * np.max(np.abs(ref.Z))
    assert set(tm) == {"permutation", "elimination", "condensation", "reduced", "backtransform", "total"}


@pytest.mark.parametrize("case", ["grid64", "hex8_force"])
def test_cpp_restatement_shift_invert_nodes(case):
    """Nodes taking the reference's shift-invert Lanczos branch (nnz/n^2 <
    0.15, n >= 200): the 64 x 64 grid of the reference's regression case."""
    if case == "grid64":
        p, o = cases.grid_graph_2d(64, 64), dict(nev=50, nLevels=4, leafSize=1000)
    else:
        p, o = cases.grid_graph_2d(40, 40), dict(nev=30, nLevels=2, leafSize=400)
    _, t = recursive_bisection(p.K, p.M, o["nLevels"], o["leafSize"])
    ref = R.amls_solve_ref(p.K, p.M, Tree.from_arrays(**t), R.OptionsRef(silMode=0, **o))
    th, Z, pp, pa, tm = cpu.solve(p.K, p.M, t, o["nev"], threads=4)
    assert pp == ref.p and pa == ref.p_passA
    assert np.max(np.abs(th - ref.theta) / ref.theta) < 1e-10
