"""Per-element eigenvalue sensitivities (adjoint kernel) against the gradient
formed from reference (LAPACK) eigenvectors and against central finite
differences of exact eigenvalues (h = 1e-6, 20 random parameters), both to
1e-6 relative."""
import numpy as np
import pytest
import torch

from amls_b200 import AmlsOptions, cases
from amls_b200.autograd import WeightedEigenvalueSum
from oracle import amls_ref as R

pytestmark = pytest.mark.gpu

OPT = dict(nev=12, nLevels=3, leafSize=120, refine=3, refineTol=1e-12)


def _exact(p, E, rho, nev):
    K = cases._assemble(p.dofmap, p.Kbar, E, p.n).toarray()
    M = cases._assemble(p.dofmap, p.Mbar, rho, p.n).toarray()
    w, V = R.LapackDense.solve_all(K, M)
    return w[:nev], V[:, :nev]


def test_sensitivities_match_reference_eigenvector_gradient(solver):
    p = cases.hex_pencil(5, 5, 5, 1, seed=9)
    sol = solver.solve(p.K, p.M, AmlsOptions(**OPT))
    sens = solver.sensitivities(p, per_mode=True)
    lam, X = _exact(p, p.E, p.rho, OPT["nev"])
    assert np.max(np.abs(sol.theta - lam) / lam) < 1e-9
    Xe = np.where(p.dofmap[:, :, None] >= 0, X[np.maximum(p.dofmap, 0)], 0.0)  # nelem x nd x nev
    dE_ref = np.einsum("eik,ij,ejk->ek", Xe, p.Kbar, Xe)
    dR_ref = -lam[None, :] * np.einsum("eik,ij,ejk->ek", Xe, p.Mbar, Xe)
    simple = sens["simple"]
    assert simple.sum() >= OPT["nev"] - 2
    for a, b in ((sens["dE"], dE_ref), (sens["dRho"], dR_ref)):
        a, b = a[:, simple], b[:, simple]
        assert np.max(np.abs(a - b)) < 1e-6 * np.max(np.abs(b))
    # non-simple modes are flagged with NaN
    assert np.all(np.isnan(sens["dE"][:, ~simple]))


def test_gradient_matches_central_differences(solver):
    p = cases.hex_pencil(4, 4, 5, 1, seed=12)
    rng = np.random.default_rng(3)
    w = rng.uniform(0.0, 1.0, OPT["nev"])
    E = torch.tensor(p.E, requires_grad=True)
    rho = torch.tensor(p.rho, requires_grad=True)
    f = WeightedEigenvalueSum.apply(E, rho, solver, p, w, AmlsOptions(**OPT))
    f.backward()
    gE, gR = E.grad.numpy(), rho.grad.numpy()
    lam0, _ = _exact(p, p.E, p.rho, OPT["nev"])
    gaps = np.minimum(np.abs(np.diff(lam0, prepend=-1e300)), np.abs(np.diff(lam0, append=1e300)))
    simple = gaps > 1e-6 * lam0
    h = 1e-6
    nelem = len(p.E)
    picks = rng.choice(2 * nelem, size=20, replace=False)
    for q in picks:
        which, e = divmod(int(q), nelem)
        base = (p.E if which == 0 else p.rho)
        step = h * base[e]
        vals = []
        for sgn in (+1, -1):
            Ev, rv = p.E.copy(), p.rho.copy()
            (Ev if which == 0 else rv)[e] += sgn * step
            lam, _ = _exact(p, Ev, rv, OPT["nev"])
            vals.append(np.dot(w[simple], lam[simple]))
        fd = (vals[0] - vals[1]) / (2 * step)
        ad = (gE if which == 0 else gR)[e]
        scale = max(abs(fd), 1e-3 * np.max(np.abs(gE if which == 0 else gR)))
        assert abs(ad - fd) <= 1e-6 * scale + 1e-9, (which, e, ad, fd)
