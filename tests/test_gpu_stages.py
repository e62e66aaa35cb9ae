"""The stage-by-stage C ABI (amls_eliminate, amls_condense, amls_reduced_eig,
amls_backtransform, amls_refine): driving the reference's two-pass policy by
hand (solver.cpp:246-266) gives the eigenvalues of amls_solve, and the
oracle's pass quantities (p, kept counts, local eigenvalues)."""
import numpy as np
import pytest

from amls_b200 import AmlsOptions, cases
from oracle import amls_ref as R

from .helpers import oracle_solve, rel_err, residuals

pytestmark = pytest.mark.gpu


def test_two_pass_by_hand_matches_solve(solver):
    p = cases.hex_pencil(5, 5, 5, 1, seed=1)
    o = dict(nev=20, nLevels=3, leafSize=100)
    whole = solver.solve(p.K, p.M, AmlsOptions(**o))
    solver.analyze(p.K, p.M, AmlsOptions(**o))
    t = solver.tree()
    N = len(t["parent"])
    solver.eliminate(p.K, p.M)
    k0 = max(4, -(-3 * 20 // N))
    pa = solver.condense("fixed", k=k0)
    kA, muA = solver.pass_modes()
    assert pa == int(kA.sum()) and np.all(kA <= np.minimum(k0, t["size"]))
    wA = solver.reduced_eig(20, vectors=False)
    cut = 2.0 * wA[19]
    pb = solver.condense("threshold", lambda_cut=cut)
    kB, muB = solver.pass_modes()
    assert pb == int(kB.sum()) and np.all(muB <= cut * (1 + 1e-12))
    th = solver.reduced_eig(20)
    Z = solver.backtransform()
    assert pb == whole.p
    assert rel_err(th, whole.theta) < 1e-12
    assert Z.shape == (p.n, 20)
    assert residuals(p.K, p.M, th, Z).max() < 10 * residuals(p.K, p.M, whole.theta, whole.Z).max() + 1e-12
    ref = oracle_solve(p, R.OptionsRef(silMode=0, **o))
    assert pb == ref.p and rel_err(th, ref.theta) < 1e-10
    assert list(kB) == list(ref.k)


def test_refine_by_hand(solver):
    p = cases.hex_pencil(6, 6, 6, 1, seed=2)
    o = dict(nev=15, nLevels=3, leafSize=150, refine=3)
    solver.analyze(p.K, p.M, AmlsOptions(**o))
    solver.eliminate(p.K, p.M)
    solver.condense("fixed", k=12)
    solver.reduced_eig(40)
    solver.backtransform()
    th, Z, it = solver.refine(15)
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    assert it >= 1
    assert rel_err(th, wr[:15]) < 1e-8
    assert residuals(p.K, p.M, th, Z).max() < 1e-6


def test_stage_order_enforced(solver):
    p = cases.hex_pencil(3, 3, 3, 1, seed=4)
    solver.analyze(p.K, p.M, AmlsOptions(nev=5, nLevels=2, leafSize=30))
    with pytest.raises(ValueError):
        solver.condense("fixed", k=3)          # before eliminate
    solver.eliminate(p.K, p.M)
    with pytest.raises(ValueError):
        solver.backtransform()                 # before the reduced solve
