"""A batch of independent pencils in one launch sequence (the uneven-batch
workload: 8-node hex boxes a x b x c, a, b, c ~ U{4..12}, nev 10): every
pencil gets the reference's own solve - its own partition, two-pass
truncation and reduced problem - so its theta must equal the oracle's on
that pencil alone (1e-10 relative) and the single-pencil GPU solve's."""
import numpy as np
import pytest

from amls_b200 import AmlsOptions, cases
from oracle import amls_ref as R

from .helpers import oracle_solve, rel_err, residuals

pytestmark = pytest.mark.gpu


def test_small_batch_matches_single_solves_and_oracle(solver):
    ps = cases.batch_pencils(6, seed=3, lo=3, hi=6)
    o = dict(nev=10, nLevels=3, leafSize=100)
    sols = solver.solve_batch([p.K for p in ps], [p.M for p in ps], AmlsOptions(**o))
    assert len(sols) == len(ps)
    for p, sb in zip(ps, sols):
        one = solver.solve(p.K, p.M, AmlsOptions(**o))
        ref = oracle_solve(p, R.OptionsRef(silMode=0, **o))
        assert len(sb.theta) == 10
        assert rel_err(sb.theta, one.theta) < 1e-10
        assert rel_err(sb.theta, ref.theta) < 1e-10
        r = residuals(p.K, p.M, sb.theta, sb.Z)
        rr = residuals(p.K, p.M, ref.theta, ref.Z)
        assert np.all(r < 10 * rr + 1e-12)
        mn = np.einsum("ij,ij->j", sb.Z, p.M @ sb.Z)
        assert np.allclose(mn, 1.0, atol=1e-12)


def test_uneven_batch_256(solver):
    """The full uneven batch: 256 pencils of 300 - 6,084 DOF, nev 10 each,
    default AMLS options.  Every pencil's theta equals the single-pencil GPU
    solve; eight pencils drawn at random also equal the oracle's."""
    ps = cases.batch_pencils(256, seed=0)
    o = dict(nev=10, nLevels=6, leafSize=500)
    sols = solver.solve_batch([p.K for p in ps], [p.M for p in ps],
                              AmlsOptions(recoverVectors=False, **o))
    worst = 0.0
    for p, sb in zip(ps, sols):
        one = solver.solve(p.K, p.M, AmlsOptions(recoverVectors=False, **o))
        worst = max(worst, rel_err(sb.theta, one.theta))
    assert worst < 1e-10
    rng = np.random.default_rng(7)
    for q in rng.choice(len(ps), size=8, replace=False):
        ref = oracle_solve(ps[q], R.OptionsRef(silMode=0, recoverVectors=False, **o))
        assert rel_err(sols[q].theta, ref.theta) < 1e-10, q


def test_batch_rejects_refinement_and_coupled_pencils(solver):
    ps = cases.batch_pencils(2, seed=1, lo=3, hi=4)
    with pytest.raises(ValueError):
        solver.solve_batch([p.K for p in ps], [p.M for p in ps], AmlsOptions(nev=5, refine=3))
