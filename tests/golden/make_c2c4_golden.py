"""Golden vectors for the precision workload (27-node hex 7^3, 9,450 DOF,
nev 100), the differentiation workload (27-node hex 10^3, 26,460 DOF,
2,000 element parameters, nev 50) and the small workload (8-node hex 12^3,
6,084 DOF, nev 20), generated on the CPU:

  c1_exact.npz   the 20 smallest exact eigenvalues of the small workload
                 (scipy ARPACK, sigma = 0, tol 1e-14);
  c2_oracle.npz  the oracle's AMLS output (theta, p, p of pass A, perm) with
                 the reference's default local eigensolver choice (silMode 0)
                 at nLevels 6, leafSize 500, eta 2;
  c2_exact.npz   the 100 smallest exact eigenvalues by shift-invert Lanczos
                 (scipy ARPACK, sigma = 0, tol 1e-14): the reference's
                 ReferenceSolver takes its Spectra shift-invert path above
                 5,000 DOF (src/reference/reference_solver.cpp:39-94);
  c4_grad.npz    for the weighted sum f = sum_k w_k lambda_k over the simple
                 modes (relative gap > 1e-6, w_k ~ U[0, 1] from seed 4):
                 the exact 50 eigenvalues, the gradient of f over all 1,000
                 E_e and 1,000 rho_e formed from the reference eigenvectors
                 (ARPACK, tol 1e-14), and central finite differences with
                 h = 1e-6 on 20 random parameters.

Finite differences: each picked parameter is moved by +h and -h and both
perturbed pencils are solved from scratch (ARPACK, tol 1e-14).  The central
difference quotient (f(+h) - f(-h)) / 2h is then evaluated two ways:
  fd_sub  subtracting the two sets of eigenvalues (loses ~9 of the 16
          digits to cancellation: f(+h) - f(-h) is ~1e-9 f);
  fd      the same quotient without cancellation, through the exact
          identity of two eigenpairs of pencils that differ in one element:
            K_+ x_+ = l_+ M x_+,  K_- x_- = l_- M x_-
            =>  (l_+ - l_-) x_-^T M x_+ = x_-^T (K_+ - K_-) x_+
          (E_e step: K_+ - K_- = 2h Kbar_e; rho_e step: M differs, and
          l_+ (c + h d) = l_- (c - h d) with c = x_-^T M x_+,
          d = x_-^T Mbar_e x_+).  Both use only the perturbed eigenpairs.

Run from the repository root (takes tens of minutes):
  python tests/golden/make_c2c4_golden.py [c1|c2|c4|both]
"""
import os
import sys
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from amls_b200 import cases  # noqa: E402
from oracle import amls_ref as R  # noqa: E402
from tests.helpers import partition  # noqa: E402

C4_NEV = 50
C4_H = 1e-6
C4_PICKS = 20


def _eigsh(K, M, k):
    w, V = spla.eigsh(sp.csc_matrix(K), k=k, M=sp.csc_matrix(M), sigma=0.0, which="LM",
                      ncv=min(K.shape[0], 3 * k + 20), tol=1e-14)
    o = np.argsort(w)
    w, V = w[o], V[:, o]
    # M-normalise (ARPACK returns M-orthonormal vectors up to rounding)
    V = V / np.sqrt(np.einsum("ij,ij->j", V, M @ V))[None, :]
    return w, V


def simple_mask(lam, tol=1e-6):
    gaps = np.minimum(np.abs(np.diff(lam, prepend=-1e300)), np.abs(np.diff(lam, append=1e300)))
    return gaps > tol * np.abs(lam)


def element_forms(p, X, mat):
    """x_{k,e}^T A x_{k,e} for every element e and column k of X."""
    Xe = np.where(p.dofmap[:, :, None] >= 0, X[np.maximum(p.dofmap, 0)], 0.0)
    return np.einsum("eik,ij,ejk->ek", Xe, mat, Xe)


def cross_form(p, e, A, Xm, Xp):
    """x_-^T A_e x_+ per mode, A_e the element matrix of element e."""
    d = p.dofmap[e]
    keep = d >= 0
    a = Xm[d[keep]]
    b = Xp[d[keep]]
    Ak = A[np.ix_(keep, keep)]
    return np.einsum("ik,ij,jk->k", a, Ak, b)


def c1():
    p = cases.config_pencil("C1", seed=0)
    w, _ = _eigsh(p.K, p.M, 20)
    print("c1 exact", w[:3], flush=True)
    np.savez(os.path.join(HERE, "c1_exact.npz"), theta=w)


def c2():
    p = cases.config_pencil("C2", seed=0)
    perm, tree = partition(p, 6, 500)
    t = time.time()
    s = R.amls_solve_ref(p.K, p.M, tree, R.OptionsRef(nev=100, nLevels=6, leafSize=500, silMode=0,
                                                       recoverVectors=False))
    print("c2 oracle", time.time() - t, "p", s.p, "pA", s.p_passA, flush=True)
    np.savez(os.path.join(HERE, "c2_oracle.npz"), theta=s.theta, p=s.p, p_passA=s.p_passA,
             perm=perm, lambda_cut=s.lambda_cut)
    t = time.time()
    w, _ = _eigsh(p.K, p.M, 100)
    print("c2 exact", time.time() - t, w[:3], flush=True)
    np.savez(os.path.join(HERE, "c2_exact.npz"), theta=w)


def c4():
    p = cases.config_pencil("C4", seed=0)
    nelem = len(p.E)
    rng = np.random.Generator(np.random.PCG64(4))
    wts = rng.uniform(0.0, 1.0, C4_NEV)
    picks = rng.choice(2 * nelem, size=C4_PICKS, replace=False)
    t = time.time()
    lam, X = _eigsh(p.K, p.M, C4_NEV)
    print("c4 base", time.time() - t, lam[:3], flush=True)
    simple = simple_mask(lam)
    ws = np.where(simple, wts, 0.0)
    dE = element_forms(p, X, p.Kbar)                         # nelem x nev
    dR = -lam[None, :] * element_forms(p, X, p.Mbar)
    gE = dE @ ws
    gR = dR @ ws
    fd = np.zeros(C4_PICKS)
    fd_sub = np.zeros(C4_PICKS)
    for t_, q in enumerate(picks):
        which, e = divmod(int(q), nelem)
        sols = []
        for sgn in (+1.0, -1.0):
            Ev, rv = p.E.copy(), p.rho.copy()
            (Ev if which == 0 else rv)[e] += sgn * C4_H
            K = cases._assemble(p.dofmap, p.Kbar, Ev, p.n)
            M = cases._assemble(p.dofmap, p.Mbar, rv, p.n)
            sols.append((_eigsh(K, M, C4_NEV), M))
        (lp, Xp), Mp = sols[0]
        (lm, Xm), Mm = sols[1]
        fd_sub[t_] = np.dot(ws, lp - lm) / (2 * C4_H)
        if which == 0:
            c = np.einsum("ik,ik->k", Xm, Mm @ Xp)           # M is the same in both
            diff = 2 * C4_H * cross_form(p, e, p.Kbar, Xm, Xp) / c
        else:
            Mbase = cases._assemble(p.dofmap, p.Mbar, p.rho, p.n)
            c = np.einsum("ik,ik->k", Xm, Mbase @ Xp)
            d = cross_form(p, e, p.Mbar, Xm, Xp)
            diff = -C4_H * d * (lp + lm) / c
        fd[t_] = np.dot(ws, diff) / (2 * C4_H)
        g = (gE if which == 0 else gR)[e]
        print(f"c4 fd {t_} param {'E' if which == 0 else 'rho'}[{e}]: grad {g:.12e} fd {fd[t_]:.12e} "
              f"sub {fd_sub[t_]:.6e} rel {abs(g - fd[t_]) / abs(fd[t_]):.2e}", flush=True)
    np.savez(os.path.join(HERE, "c4_grad.npz"), lam=lam, weights=wts, simple=simple, gE=gE, gR=gR,
             picks=picks, fd=fd, fd_sub=fd_sub, h=C4_H)


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "both"
    if which == "c1":
        c1()
    if which in ("c2", "both"):
        c2()
    if which in ("c4", "both"):
        c4()
