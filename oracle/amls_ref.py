"""CPU restatement of the reference AMLS numerics (test infrastructure: the oracle).

This module is the parity checker and the CPU baseline; the product never
imports it.  It restates, in numpy/scipy float64, the algorithm of
yuesewuta/AMLS after partitioning:

* ``GaussianEliminationRef``   src/amls/gaussian_elimination.cpp:458-826
  (factorNode_, solveXYAnc_, makeWX_, schurK*/cong* tasks, applyNodeB_),
  sequential post-order as in ``run(1)`` (:828-838).  Column restriction
  semantics of ColCompOps (src/linalg/colcomp.hpp:238-354) are kept: X_a and
  Y_a are solved only for the nonzero columns of K_{i,a} / M_{i,a} and the
  products update only those columns; targets are stored dense.
* ``EigenpairSolverRef``       src/amls/eigenpair_solver.hpp:19-85 (dense
  dsygvx vs. shift-invert Lanczos by the nnz/n^2 < 0.15 and n >= 200 rule),
  ``LapackDense``              src/linalg/dense_eigensolver.cpp:11-133
  (scipy's LAPACK dsygvd / dsygvx with itype 1, uplo 'L', abstol 0),
  ``sil_*``                    src/amls/shift_invert_lanczos.hpp:32-203.
* truncation policies          src/amls/spectral_truncation.hpp:35-88.
* ``SubspaceCondensationRef``  src/amls/subspace_condensation.cpp:18-319.
* ``amls_solve_ref``           src/amls/solver.cpp:100-319.

Third-party arithmetic: LAPACK dsygvd/dsygvx (reference: netlib LAPACK,
unpinned) is scipy's bundled LAPACK; Eigen's SimplicialLDLT/LDLT
(unpinned) becomes a dense Cholesky (scipy.linalg.cho_factor) - the same
factorisation up to rounding for SPD blocks; Eigen's random start vector of
the Lanczos (std::srand(12345), Vec::Random) is restated for Eigen 3.4 over
the Microsoft C runtime's rand() (``reference_start_vector``).
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np
import scipy.linalg as sla
import scipy.linalg.lapack as lapack
import scipy.sparse as sp

from .tree import Tree


class NotSPDError(RuntimeError):
    """Non-positive pivot (reference: sparse_direct.cpp:17-22, 48-53)."""


# --------------------------------------------------------------------------
# dense generalized eigensolver (dense_eigensolver.cpp)
# --------------------------------------------------------------------------

class LapackDense:
    """dsygvd / dsygvx wrappers with the reference's arguments."""

    @staticmethod
    def solve_all(K, M):
        n = K.shape[0]
        if n == 0:
            return np.zeros(0), np.zeros((0, 0))
        w, v, info = lapack.dsygvd(np.asfortranarray(K), np.asfortranarray(M), itype=1,
                                   jobz="V", uplo="L")
        if info != 0:
            raise RuntimeError(f"dsygvd failed, info={info}")
        return w, v

    @staticmethod
    def solve_interval(K, M, lo, hi):
        """(lo, hi] by value (dense_eigensolver.cpp:44-86)."""
        n = K.shape[0]
        if n == 0 or not (hi > lo):
            return np.zeros(0), np.zeros((n, 0))
        w, z, m, ifail, info = lapack.dsygvx(np.asfortranarray(K), np.asfortranarray(M), itype=1,
                                             jobz="V", range="V", uplo="L", vl=lo, vu=hi,
                                             abstol=0.0, lwork=max(1, 8 * n))
        if info != 0:
            raise RuntimeError(f"dsygvx failed, info={info}")
        return w[:m].copy(), z[:, :m].copy()

    @staticmethod
    def solve_index(K, M, il, iu):
        """[il, iu], 1-based (dense_eigensolver.cpp:88-133)."""
        n = K.shape[0]
        if n == 0 or iu < il:
            return np.zeros(0), np.zeros((n, 0))
        iu = min(iu, n)
        w, z, m, ifail, info = lapack.dsygvx(np.asfortranarray(K), np.asfortranarray(M), itype=1,
                                             jobz="V", range="I", uplo="L", il=il, iu=iu,
                                             abstol=0.0, lwork=max(1, 8 * n))
        if info != 0:
            raise RuntimeError(f"dsygvx failed, info={info}")
        return w[:m].copy(), z[:, :m].copy()


# --------------------------------------------------------------------------
# shift-invert Lanczos (shift_invert_lanczos.hpp)
# --------------------------------------------------------------------------

def msvcrt_rand(seed: int, count: int) -> np.ndarray:
    """std::rand() after std::srand(seed) in the Microsoft C runtime that the
    reference's documented toolchain (MSYS2 mingw64, docs/环境与构建说明.md:4)
    links: state <- 214013 state + 2531011 (mod 2^32), value
    (state >> 16) & 0x7fff, RAND_MAX = 0x7fff."""
    out = np.empty(count, np.int64)
    x = seed & 0xFFFFFFFF
    for i in range(count):
        x = (x * 214013 + 2531011) & 0xFFFFFFFF
        out[i] = (x >> 16) & 0x7FFF
    return out


def reference_start_vector(n: int, seed: int = 12345) -> np.ndarray:
    """The Lanczos start vector of shift_invert_lanczos.hpp:49-50:
    std::srand(seed) then Eigen's Vec::Random(n), which in Eigen 3.4 draws
    -1 + 2 rand() / RAND_MAX per entry in order.  (Eigen 3.4 is an
    assumption: the reference leaves its version unpinned, and later Eigen
    releases draw random bits differently.)"""
    return -1.0 + 2.0 * msvcrt_rand(seed, n).astype(np.float64) / 32767.0


class _SIL:
    """M-inner-product Lanczos on C = (K - sigma M)^-1 M with full double
    reorthogonalisation (shift_invert_lanczos.hpp:32-122)."""

    def __init__(self, Kd, Md, sigma):
        self.n = Kd.shape[0]
        self.shift = sigma
        # Eigen's sparseView(1e-14) keeps |x| > 1e-14 * dummy_precision (1e-12)
        Ks = np.where(np.abs(Kd) > 1e-26, Kd, 0.0)
        self.M = np.where(np.abs(Md) > 1e-26, Md, 0.0)
        A = Ks - sigma * self.M
        try:
            self.fact = sla.cho_factor(A, lower=True, check_finite=False)
        except np.linalg.LinAlgError as e:
            raise NotSPDError("SIL: factorisation failed (not SPD)") from e

    def _applyC(self, x):
        return sla.cho_solve(self.fact, self.M @ x, check_finite=False)

    def iterate(self, ncv, seed=12345):
        ncv = min(ncv, self.n)
        alpha = np.zeros(ncv)
        beta = np.zeros(ncv)
        Q = np.zeros((self.n, ncv))
        q0 = reference_start_vector(self.n, seed)
        q0 /= math.sqrt(max(q0 @ (self.M @ q0), 1e-300))
        Q[:, 0] = q0
        m = 0
        for j in range(ncv):
            w = self._applyC(Q[:, j])
            alpha[j] = Q[:, j] @ (self.M @ w)
            for _ in range(2):
                for l in range(j + 1):
                    w = w - (Q[:, l] @ (self.M @ w)) * Q[:, l]
            bj = math.sqrt(max(w @ (self.M @ w), 0.0))
            m = j + 1
            if bj < 1e-13 or m == ncv:
                break                      # beta[j] stays 0 (reference :67-69)
            beta[j] = bj
            Q[:, j + 1] = w / bj
        self.m = m
        self.beta = beta
        T = np.diag(alpha[:m]) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
        self.nu, self.S = np.linalg.eigh(T)
        self.Q = Q[:, :m]
        return m

    def lam(self, j):
        return 1.0 / self.nu[j] + self.shift

    def res(self, j):
        bm = self.beta[self.m - 1] if self.m > 1 else 0.0
        return abs(bm * self.S[self.m - 1, j])

    def ritz(self, j):
        return self.Q @ self.S[:, j]


def sil_solve_interval(Kd, Md, lo, hi, tol=1e-9):
    """shift_invert_lanczos.hpp:126-168."""
    n = Kd.shape[0]
    scale = float(np.max(np.abs(np.diag(Kd)))) if n else 0.0
    lo_sane = lo if lo > -1e100 else 0.0
    sigma = min(0.0, lo_sane) - max(1e-10, 1e-9 * (scale if scale > 0 else 1.0))
    lz = _SIL(Kd, Md, sigma)
    ncv = min(n, 96)
    cap = min(n, 1536)
    while True:
        m = lz.iterate(ncv)
        cnt = sum(1 for j in range(m) if lz.lam(j) <= hi)
        if cnt < m and cnt > 0 and lz.res(cnt - 1) <= tol * max(1.0, lz.nu[m - 1]):
            break
        if ncv >= cap or m < ncv:
            break
        ncv = min(cap, ncv * 2)
    pick = [j for j in range(lz.m)
            if not (lz.lam(j) > hi or lz.lam(j) <= lo)
            and lz.res(j) <= 100 * tol * max(1.0, lz.nu[lz.m - 1])]
    w = np.array([lz.lam(j) for j in pick])
    V = np.stack([lz.ritz(j) for j in pick], axis=1) if pick else np.zeros((n, 0))
    return w, V


def sil_solve_index(Kd, Md, il, iu, tol=1e-10):
    """shift_invert_lanczos.hpp:171-203."""
    n = Kd.shape[0]
    k = iu - il + 1
    scale = float(np.max(np.abs(np.diag(Kd)))) if n else 0.0
    sigma = -max(1e-10, 1e-9 * (scale if scale > 0 else 1.0))
    lz = _SIL(Kd, Md, sigma)
    cap = min(n, 1536)
    ncv = min(n, max(4 * k + 16, 48))
    while True:
        m = lz.iterate(ncv)
        want = min(k, m)
        ok = all(lz.res(m - 1 - t) <= tol * max(1.0, lz.nu[m - 1]) for t in range(want))
        if ok or ncv >= cap or m < ncv:
            break
        ncv = min(cap, ncv * 2)
    m = lz.m
    kk = min(k, m)
    w = np.array([lz.lam(m - 1 - t) for t in range(kk)])
    V = np.stack([lz.ritz(m - 1 - t) for t in range(kk)], axis=1) if kk else np.zeros((n, 0))
    return w, V


class EigenpairSolverRef:
    """Local eigensolver dispatch (eigenpair_solver.hpp:19-85).
    sil_mode: 0 auto by sparsity, 1 force SIL, -1 force dense."""

    def __init__(self, sil_mode: int = 0):
        self.sil_mode = sil_mode

    def _use_sil(self, K):
        if self.sil_mode > 0:
            return True
        if self.sil_mode < 0:
            return False
        n = K.shape[0]
        if n < 200:
            return False
        return np.count_nonzero(K) < 0.15 * n * n

    def solve_all(self, K, M):
        return LapackDense.solve_all(K, M)

    def solve_interval(self, K, M, lo, hi):
        if self._use_sil(K):
            w, V = sil_solve_interval(K, M, lo, hi)
            if w.size == 0:
                w, V = LapackDense.solve_interval(K, M, lo, hi)
            return w, V
        return LapackDense.solve_interval(K, M, lo, hi)

    def solve_index(self, K, M, il, iu):
        n = K.shape[0]
        if il == 1 and self._use_sil(K):
            k = iu - il + 1
            if k < (n * 4) // 5:
                w, V = sil_solve_index(K, M, il, iu)
                if w.size == k:
                    return w, V
        return LapackDense.solve_index(K, M, il, iu)


# --------------------------------------------------------------------------
# truncation policies (spectral_truncation.hpp)
# --------------------------------------------------------------------------

class ThresholdTruncation:
    def __init__(self, lambda_cut):
        self.cut = lambda_cut

    def select(self, w, max_keep):
        k = 0
        while k < max_keep and k < len(w) and w[k] <= self.cut:
            k += 1
        return k

    def interval_hint(self):
        return (-1e300, self.cut)

    def index_hint(self):
        return None


class FixedCountTruncation:
    def __init__(self, k):
        self.k = k

    def select(self, w, max_keep):
        if self.k <= 0:
            return max_keep
        return min(self.k, max_keep)

    def interval_hint(self):
        return None

    def index_hint(self):
        return (1, self.k) if self.k > 0 else None


# --------------------------------------------------------------------------
# Gaussian elimination (gaussian_elimination.cpp)
# --------------------------------------------------------------------------

def _nonzero_rows(B) -> np.ndarray:
    """Nonzero rows of a coupling block = nonzero columns of its transpose,
    i.e. the right-hand-side columns the reference solves for
    (gaussian_elimination.cpp:517-551 buildSub / :552-563 buildSubDense)."""
    if sp.issparse(B):
        Bc = sp.csc_matrix(B)
        return np.unique(Bc.indices).astype(np.int64)
    return np.nonzero(np.any(B != 0.0, axis=1))[0]


def _rows(B, idx):
    return B[idx, :].toarray() if sp.issparse(B) else B[idx, :]


class GaussianEliminationRef:
    """Post-order block elimination of K with M congruence, on the permuted
    pencil (gaussian_elimination.cpp:458-838)."""

    def __init__(self, K: sp.csr_matrix, M: sp.csr_matrix, tree: Tree):
        self.tree = tree
        self.N = tree.n_nodes
        self.order = tree.post_order()
        self.off = [0] * self.N
        self.size = [0] * self.N
        acc = 0
        for i in self.order:                      # precompute_ :183-194
            self.off[i] = acc
            self.size[i] = len(tree.indices[i])
            acc += self.size[i]
        self.level = tree.levels()
        self.max_level = max(self.level)
        self.by_level = [[i for i in self.order if self.level[i] == l]
                         for l in range(self.max_level + 1)]
        Kc, Mc = sp.csc_matrix(K), sp.csc_matrix(M)
        self._Kc, self._Mc = Kc, Mc
        self.orig_kdiag, self.orig_mdiag = {}, {}
        self.orig_kcoup, self.orig_mcoup = {}, {}
        for i in range(self.N):
            o, n = self.off[i], self.size[i]
            self.orig_kdiag[i] = Kc[o:o + n, o:o + n].toarray()
            self.orig_mdiag[i] = Mc[o:o + n, o:o + n].toarray()
            for a in tree.ancestors(i):
                oa, na = self.off[a], self.size[a]
                self.orig_kcoup[(a, i)] = sp.csc_matrix(Kc[oa:oa + na, o:o + n])
                self.orig_mcoup[(a, i)] = sp.csc_matrix(Mc[oa:oa + na, o:o + n])
        self.reset_blocks()

    def reset_blocks(self):
        self.kdiag, self.mdiag = {}, {}
        self.kcoup, self.mcoup = {}, {}
        self.factors = [None] * self.N
        self.timing = {}

    # targets (kDiagTarget_ :421-432, kCoupTarget_ :364-390)
    def _kdiag_t(self, a):
        if a not in self.kdiag:
            self.kdiag[a] = self.orig_kdiag[a].copy()
        return self.kdiag[a]

    def _mdiag_t(self, a):
        if a not in self.mdiag:
            self.mdiag[a] = self.orig_mdiag[a].copy()
        return self.mdiag[a]

    def _kcoup_t(self, hi, lo):
        if (hi, lo) not in self.kcoup:
            self.kcoup[(hi, lo)] = self.orig_kcoup[(hi, lo)].toarray()
        return self.kcoup[(hi, lo)]

    def _mcoup_t(self, hi, lo):
        if (hi, lo) not in self.mcoup:
            self.mcoup[(hi, lo)] = self.orig_mcoup[(hi, lo)].toarray()
        return self.mcoup[(hi, lo)]

    # read access for the condensation (get-value API, .hpp:113-153)
    def is_leaf(self, i):
        return self.tree.is_leaf(i)

    def k_hat(self, i):
        return self.orig_kdiag[i] if self.is_leaf(i) else self.kdiag[i]

    def m_hat(self, i):
        return self.orig_mdiag[i] if self.is_leaf(i) else self.mdiag[i]

    def k_coupling(self, a, i):
        if self.is_leaf(i):
            return self.orig_kcoup[(a, i)]
        return self.kcoup.get((a, i), np.zeros((self.size[a], self.size[i])))

    def m_coupling(self, a, i):
        if self.is_leaf(i):
            return self.orig_mcoup[(a, i)]
        return self.mcoup.get((a, i), np.zeros((self.size[a], self.size[i])))

    def solve_factor(self, i, B):
        return sla.cho_solve(self.factors[i], B, check_finite=False)

    def _factor(self, i):
        A = self.orig_kdiag[i] if self.is_leaf(i) else self._kdiag_t(i)
        try:
            c, low = sla.cho_factor(A, lower=True, check_finite=False)
        except np.linalg.LinAlgError as e:
            raise NotSPDError(f"node {i}: non-positive pivot") from e
        if not np.all(np.isfinite(np.diag(c))) or np.any(np.diag(c) <= 0):
            raise NotSPDError(f"node {i}: non-positive pivot")
        self.factors[i] = (c, low)

    def eliminate_node(self, i):
        anc = self.tree.ancestors(i)
        t0 = time.perf_counter()
        self._factor(i)
        self.timing["factor"] = self.timing.get("factor", 0.0) + time.perf_counter() - t0
        if not anc:
            return
        leaf = self.is_leaf(i)
        W = self.orig_mdiag[i] if leaf else self._mdiag_t(i)
        Kc = {a: self.k_coupling(a, i) for a in anc}          # K_{a,i} (n_a x n_i)
        Mc = {a: self.m_coupling(a, i) for a in anc}
        X, Y, WX = {}, {}, {}
        t1 = time.perf_counter()
        for a in anc:                                          # solveXYAnc_ :510-598
            xi = _nonzero_rows(Kc[a])
            X[a] = (xi, self.solve_factor(i, _rows(Kc[a], xi).T) if xi.size else None)
            yi = _nonzero_rows(Mc[a])
            Y[a] = (yi, self.solve_factor(i, _rows(Mc[a], yi).T) if yi.size else None)
            # makeWX_ :653-676: K^-1 (M^ X) over X's nonzero columns
            WX[a] = (xi, self.solve_factor(i, W @ X[a][1]) if xi.size else None)
        t2 = time.perf_counter()
        self.timing["solve"] = self.timing.get("solve", 0.0) + t2 - t1
        # K Schur (schurKDiagTask_ :678-696, schurKCoupTask_ :698-715)
        for a in anc:
            xi, Xs = X[a]
            if Xs is not None:
                self._kdiag_t(a)[:, xi] -= Kc[a] @ Xs
        for p in range(len(anc)):
            for q in range(p + 1, len(anc)):
                hi, lo = anc[q], anc[p]
                xi, Xs = X[lo]
                tgt = self._kcoup_t(hi, lo)
                if Xs is not None:
                    tgt[:, xi] -= Kc[hi] @ Xs
        # M congruence (congDiagTask_ :717-743, congCoupTask_ :745-781)
        for a in anc:
            md = self._mdiag_t(a)
            yi, Ys = Y[a]
            if Ys is not None:
                T = Kc[a] @ Ys                                  # n_a x |yi|
                md[:, yi] -= T
                md[yi, :] -= T.T
            xi, WXs = WX[a]
            if WXs is not None:
                md[:, xi] += Kc[a] @ WXs
        for p in range(len(anc)):
            for q in range(p + 1, len(anc)):
                hi, lo = anc[q], anc[p]
                tgt = self._mcoup_t(hi, lo)
                yi, Ys = Y[lo]
                if Ys is not None:
                    tgt[:, yi] -= Kc[hi] @ Ys
                yh, Yh = Y[hi]
                if Yh is not None:
                    tgt[yh, :] -= (Kc[lo] @ Yh).T
                xi, WXs = WX[lo]
                if WXs is not None:
                    tgt[:, xi] += Kc[hi] @ WXs
        self.timing["update"] = self.timing.get("update", 0.0) + time.perf_counter() - t2

    def run(self):
        self.reset_blocks()
        for i in self.order:
            self.eliminate_node(i)


# --------------------------------------------------------------------------
# subspace condensation (subspace_condensation.cpp)
# --------------------------------------------------------------------------

@dataclasses.dataclass
class CondResult:
    p: int
    proj_offset: list
    k: list
    mu: list
    Z: list
    mproj_blocks: list          # (row node, col node, block k_row x k_col)


class SubspaceCondensationRef:
    def __init__(self, ge: GaussianEliminationRef, eig: EigenpairSolverRef):
        self.ge = ge
        self.eig = eig
        self.N = ge.N

    def run(self, truncation) -> CondResult:
        """run (:18-36): all local spectra, then all projections, offsets."""
        N = self.N
        res = CondResult(0, [0] * N, [0] * N, [np.zeros(0)] * N, [np.zeros((0, 0))] * N, [])
        self.mbar = {}
        self.mbar_row = {}
        for l in range(self.ge.max_level + 1):
            self.spectral_level(truncation, l, res)
        for l in range(self.ge.max_level + 1):
            for i in self.ge.by_level[l]:
                self.project_node(i, res)
        acc = 0
        for i in range(N):                              # finalize :120-127
            res.proj_offset[i] = acc
            acc += res.k[i]
        res.p = acc
        return res

    def spectral_level(self, truncation, l, res):
        """(:45-100)"""
        for i in self.ge.by_level[l]:
            Kh = np.array(self.ge.k_hat(i), copy=True)
            Mh = np.array(self.ge.m_hat(i), copy=True)
            ih = truncation.interval_hint()
            xh = truncation.index_hint()
            if ih is not None:
                w, V = self.eig.solve_interval(Kh, Mh, ih[0], ih[1])
            elif xh is not None:
                w, V = self.eig.solve_index(Kh, Mh, xh[0], xh[1])
            else:
                w, V = self.eig.solve_all(Kh, Mh)
            ki = truncation.select(w, len(w))
            res.k[i] = ki
            if ki > 0:
                res.mu[i] = w[:ki].copy()
                res.Z[i] = V[:, :ki].copy()

    def project_node(self, i, res):
        """projectNode_ (:129-261)."""
        ge = self.ge
        anc = ge.tree.ancestors(i)
        ki = res.k[i]
        rowKK = list(self.mbar_row.get(i, []))
        if anc:
            if rowKK:                                   # mid-node column update :146-202
                RHS = np.concatenate([self.mbar[(i, kk)] for kk in rowKK], axis=1)
                Vs = ge.solve_factor(i, RHS)
                off = 0
                for kk in rowKK:
                    kc = self.mbar[(i, kk)].shape[1]
                    Vk = Vs[:, off:off + kc]
                    for a in anc:
                        self.mbar[(a, kk)] -= ge.k_coupling(a, i) @ Vk
                    off += kc
            if ki > 0:                                  # right projection init :204-232
                Zi = res.Z[i]
                Mz = ge.m_hat(i) @ Zi
                WMz = ge.solve_factor(i, Mz)
                for a in anc:
                    proj = ge.m_coupling(a, i) @ Zi - ge.k_coupling(a, i) @ WMz
                    self.mbar[(a, i)] = np.asarray(proj)
                    self.mbar_row.setdefault(a, []).append(i)
        if ki > 0:                                      # left projection :235-254
            for kk in rowKK:
                res.mproj_blocks.append((i, kk, res.Z[i].T @ self.mbar[(i, kk)]))
        for kk in rowKK:
            del self.mbar[(i, kk)]
        self.mbar_row.pop(i, None)

    def backtransform(self, r: CondResult, Q: np.ndarray) -> np.ndarray:
        """z = L^-T S q in reverse post-order (:263-319)."""
        ge = self.ge
        m = Q.shape[1]
        n = sum(ge.size)
        z = [None] * self.N
        for i in reversed(ge.order):
            ni, ki = ge.size[i], r.k[i]
            if ki > 0:
                yi = r.Z[i] @ Q[r.proj_offset[i]:r.proj_offset[i] + ki, :]
            else:
                yi = np.zeros((ni, m))
            rhs = np.zeros((ni, m))
            for a in ge.tree.ancestors(i):
                rhs += np.asarray(ge.k_coupling(a, i).T @ z[a])
            z[i] = yi - ge.solve_factor(i, rhs)
        out = np.zeros((n, m))
        for i in range(self.N):
            out[ge.off[i]:ge.off[i] + ge.size[i], :] = z[i]
        return out


def assemble_mproj(r: CondResult) -> np.ndarray:
    """solver.cpp:71-84: I + symmetric tree blocks."""
    Mp = np.eye(r.p)
    for (ri, ci, blk) in r.mproj_blocks:
        r0, c0 = r.proj_offset[ri], r.proj_offset[ci]
        Mp[r0:r0 + blk.shape[0], c0:c0 + blk.shape[1]] = blk
        Mp[c0:c0 + blk.shape[1], r0:r0 + blk.shape[0]] = blk.T
    return Mp


def assemble_kproj(r: CondResult) -> np.ndarray:
    """solver.cpp:86-96: diag(mu)."""
    Kp = np.zeros((r.p, r.p))
    for i in range(len(r.k)):
        o = r.proj_offset[i]
        for j in range(r.k[i]):
            Kp[o + j, o + j] = r.mu[i][j]
    return Kp


def solve_projected(r: CondResult, want: int):
    """solver.cpp:145-161."""
    if r.p <= 0:
        raise RuntimeError("reduced problem is empty (all nodes truncated)")
    Mp = assemble_mproj(r)
    Kp = assemble_kproj(r)
    want = min(want, r.p)
    if want < r.p:
        return LapackDense.solve_index(Kp, Mp, 1, want)
    return LapackDense.solve_all(Kp, Mp)


@dataclasses.dataclass
class OptionsRef:
    """AmlsOptions (solver.hpp:18-30)."""
    nLevels: int = 6
    leafSize: int = 500
    thresholdFactor: float = 2.0
    fixedKeep: int = 0
    nev: int = 100
    denseProjectedMax: int = 5000
    shift: float = 0.0
    twoPass: bool = True
    recoverVectors: bool = True
    silMode: int = 0


@dataclasses.dataclass
class SolutionRef:
    theta: np.ndarray
    Z: np.ndarray | None
    p: int
    p_passA: int
    k: list
    timing: dict
    lambda_cut: float


def permute_symmetric(A: sp.csr_matrix, perm: np.ndarray) -> sp.csr_matrix:
    """B = P A P^T with perm[new] = old (solver.cpp:48-69)."""
    B = sp.csr_matrix(A)[perm, :][:, perm]
    B.sort_indices()
    return sp.csr_matrix(B)


def amls_solve_ref(K: sp.csr_matrix, M: sp.csr_matrix, tree: Tree, opt: OptionsRef) -> SolutionRef:
    """AmlsSolver::solve (solver.cpp:100-319) on a given partition tree."""
    if opt.nev <= 0:
        raise ValueError("nev must be positive")
    n = K.shape[0]
    if n == 0:
        raise ValueError("empty matrix")
    nev = min(opt.nev, n)
    timing = {}
    t0 = time.perf_counter()
    if opt.shift != 0.0:
        K = sp.csr_matrix(K + opt.shift * M)
    perm = tree.perm()
    Kp = permute_symmetric(K, perm)
    Mp = permute_symmetric(M, perm)
    t1 = time.perf_counter()
    timing["partition"] = t1 - t0
    ge = GaussianEliminationRef(Kp, Mp, tree)
    eig = EigenpairSolverRef(opt.silMode)
    cond = SubspaceCondensationRef(ge, eig)
    ge.run()                                    # elimination is independent of truncation
    t2 = time.perf_counter()
    timing["gauss"] = t2 - t1
    lambda_cut = -1.0
    p_a = 0
    if opt.fixedKeep > 0:
        res = cond.run(FixedCountTruncation(opt.fixedKeep))
    else:
        if not opt.twoPass:
            raise ValueError("twoPass=false with fixedKeep=0 cannot set the cut")
        N = tree.n_nodes
        k0 = max(4, (3 * nev + N - 1) // N)
        ra = cond.run(FixedCountTruncation(k0))
        p_a = ra.p
        wA, _ = solve_projected(ra, min(nev, ra.p))
        if len(wA) < nev:
            raise RuntimeError("pass A reduced problem too small (p < nev)")
        lambda_hat = wA[nev - 1]
        lambda_cut = opt.thresholdFactor * lambda_hat
        res = cond.run(ThresholdTruncation(lambda_cut))
    t3 = time.perf_counter()
    timing["condense"] = t3 - t2
    want = min(nev, res.p)
    theta, Q = solve_projected(res, want)
    t4 = time.perf_counter()
    timing["reduced"] = t4 - t3
    Z = None
    if opt.recoverVectors:
        z = cond.backtransform(res, Q)
        X = np.zeros_like(z)
        X[perm, :] = z
        MX = M @ X
        for c in range(X.shape[1]):
            mz = X[:, c] @ MX[:, c]
            X[:, c] /= math.sqrt(max(mz, 1e-300))
        Z = X
    timing["backtransform"] = time.perf_counter() - t4
    return SolutionRef(theta, Z, res.p, p_a, list(res.k), timing, lambda_cut)


# --------------------------------------------------------------------------
# exact reference eigenpairs (src/reference/reference_solver.cpp:18-95)
# --------------------------------------------------------------------------

def smallest_eigenpairs(K, M, nev, dense_max=5000):
    """Dense dsygvd for n <= dense_max, else shift-invert Lanczos at sigma = 0
    (scipy ARPACK standing in for Spectra's SymGEigsShiftSolver, tol 1e-12)."""
    n = K.shape[0]
    nev = min(nev, n)
    if n <= dense_max:
        w, V = LapackDense.solve_all(K.toarray(), M.toarray())
        return w[:nev], V[:, :nev]
    import scipy.sparse.linalg as spla
    w, V = spla.eigsh(sp.csc_matrix(K), k=nev, M=sp.csc_matrix(M), sigma=0.0, which="LM",
                      ncv=min(3 * nev + 20, n), tol=1e-12, maxiter=1000)
    o = np.argsort(w)
    return w[o], V[:, o]
