"""Per-element eigenvalue sensitivities (adjoint kernel) against the gradient
formed from reference (LAPACK / ARPACK) eigenvectors and against central
finite differences of exact eigenvalues (h = 1e-6, 20 random parameters),
both to 1e-6 relative: on small cubes (dense LAPACK for every perturbed
pencil), on a mesh with two element types, and on the differentiation
workload (27-node hex 10^3, 26,460 DOF, 2,000 parameters, nev 50) against
the golden gradient and finite differences of tests/golden/make_c2c4_golden.py."""
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


def test_sensitivities_two_element_types(solver):
    """A mesh whose elements come in two types (different element matrices):
    the adjoint kernel picks each element's matrices by its type."""
    p = cases.hex_pencil(4, 4, 5, 1, seed=21)
    nelem = len(p.E)
    et = (np.arange(nelem) % 3 == 0).astype(np.int32)         # every third element is type 1
    Kb = np.stack([p.Kbar, 1.7 * p.Kbar + 0.1 * np.diag(np.diag(p.Kbar))])
    Mb = np.stack([p.Mbar, 0.6 * p.Mbar])
    K = sum(cases._assemble(p.dofmap[et == t], Kb[t], p.E[et == t], p.n) for t in (0, 1))
    M = sum(cases._assemble(p.dofmap[et == t], Mb[t], p.rho[et == t], p.n) for t in (0, 1))
    nev = 12
    sol = solver.solve(K, M, AmlsOptions(**OPT))
    q = cases.Pencil(K, M, dofmap=p.dofmap, Kbar=Kb, Mbar=Mb, E=p.E, rho=p.rho)
    sens = solver.sensitivities(q, per_mode=True, elem_type=et)
    lam, X = R.LapackDense.solve_all(K.toarray(), M.toarray())
    lam, X = lam[:nev], X[:, :nev]
    assert np.max(np.abs(sol.theta - lam) / lam) < 1e-9
    Xe = np.where(p.dofmap[:, :, None] >= 0, X[np.maximum(p.dofmap, 0)], 0.0)
    dE_ref = np.einsum("eik,eij,ejk->ek", Xe, Kb[et], Xe)
    dR_ref = -lam[None, :] * np.einsum("eik,eij,ejk->ek", Xe, Mb[et], Xe)
    simple = sens["simple"]
    for a, b in ((sens["dE"], dE_ref), (sens["dRho"], dR_ref)):
        a, b = a[:, simple], b[:, simple]
        assert np.max(np.abs(a - b)) < 1e-6 * np.max(np.abs(b))


def test_c4_gradient_matches_golden_and_finite_differences(solver):
    """Differentiation workload (27-node hex 10^3,
    26,460 DOF, 2,000 element parameters, nev 50, w_k ~ U[0, 1], simple modes
    with relative gap > 1e-6): the adjoint gradient of sum_k w_k lambda_k
    over all E_e and rho_e equals the gradient from the reference (ARPACK)
    eigenvectors to 1e-6 relative, and the central finite differences
    (h = 1e-6) on 20 random parameters to 1e-6 relative."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c4_grad.npz"))
    p = cases.config_pencil("C4", seed=0)
    nev = 50
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=nev, nLevels=6, leafSize=500, refine=3,
                                             refineTol=1e-12))
    assert np.max(np.abs(sol.theta - g["lam"]) / g["lam"]) < 1e-9
    sens = solver.sensitivities(p, weights=g["weights"])
    assert np.array_equal(sens["simple"], g["simple"])
    for a, b in ((sens["gE"], g["gE"]), (sens["gRho"], g["gR"])):
        assert np.max(np.abs(a - b)) < 1e-6 * np.max(np.abs(b))
    nelem = len(p.E)
    for q, fd in zip(g["picks"], g["fd"]):
        which, e = divmod(int(q), nelem)
        ad = (sens["gE"] if which == 0 else sens["gRho"])[e]
        assert abs(ad - fd) <= 1e-6 * abs(fd), (which, e, ad, fd)
