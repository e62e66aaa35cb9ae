"""Host-side mirror of the reference's solver interface over the C ABI.

``AmlsSolver.solve(K, M, opt)`` corresponds to ``AmlsSolver::solve``
(src/amls/solver.cpp:100-319): same options and defaults, same exceptions
(``ValueError`` for std::invalid_argument, ``RuntimeError`` subclasses for
std::runtime_error), ``Solution`` with theta ascending, Z M-normalised in the
original ordering, the reduced size p and the phase timings.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import scipy.sparse as sp

from . import _lib


@dataclasses.dataclass
class AmlsOptions:
    """AmlsOptions (src/amls/solver.hpp:18-30)."""
    nLevels: int = 6
    leafSize: int = 500
    thresholdFactor: float = 2.0
    fixedKeep: int = 0
    nev: int = 100
    denseProjectedMax: int = 5000
    shift: float = 0.0
    twoPass: bool = True
    numThreads: int = 0
    recoverVectors: bool = True
    verbosity: int = 0
    # FP64 refinement (not in the reference): subspace iteration with the
    # elimination's exact K factorisation + Rayleigh-Ritz
    refine: int = 0            # 0 off; k >= 1: K^-1 M applications per Rayleigh-Ritz step
    refineMaxIter: int = 60
    refineExtra: int = -1
    refineTol: float = 1e-9
    # "fp64" or "mixed" (M-side AMLS products on the BF16 tensor cores, split
    # operands; not in the reference)
    precision: str = "fp64"
    # local eigensolver per node (EigenpairSolver::silMode): 0 automatic by
    # sparsity, 1 shift-invert Lanczos everywhere, -1 dense everywhere
    silMode: int = 0

    def to_c(self) -> _lib.Options:
        o = _lib.Options()
        _lib.check(_lib.lib().amls_options_default(C.byref(o)))
        o.nLevels = int(self.nLevels)
        o.leafSize = int(self.leafSize)
        o.thresholdFactor = float(self.thresholdFactor)
        o.fixedKeep = int(self.fixedKeep)
        o.nev = int(self.nev)
        o.denseProjectedMax = int(self.denseProjectedMax)
        o.shift = float(self.shift)
        o.twoPass = 1 if self.twoPass else 0
        o.numThreads = int(self.numThreads)
        o.recoverVectors = 1 if self.recoverVectors else 0
        o.verbosity = int(self.verbosity)
        o.refine = (3 if self.refine is True else int(self.refine))
        o.refineMaxIter = int(self.refineMaxIter)
        o.refineExtra = int(self.refineExtra)
        o.refineTol = float(self.refineTol)
        if self.precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {self.precision!r}")
        o.precision = 0 if self.precision == "fp64" else 1
        if int(self.silMode) not in (-1, 0, 1):
            raise ValueError("silMode must be -1, 0 or 1")
        o.silMode = int(self.silMode)
        return o


@dataclasses.dataclass
class Solution:
    theta: np.ndarray
    Z: np.ndarray | None
    p: int
    timing: dict
    info: dict


def _csr_arrays(A):
    """Row pointers (int64), columns (int32, sorted within rows) and values
    of A as CSR; a CSR input with sorted indices is used as it is (no copy),
    anything else is converted (the caller's matrix is never modified)."""
    if not (sp.issparse(A) and A.format == "csr"):
        A = sp.csr_matrix(A)
    if not A.has_sorted_indices:
        A = A.copy()
        A.sort_indices()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    return rp, ci, v


def _block_diag(As) -> sp.csr_matrix:
    """Block-diagonal CSR of square matrices (sorted indices, int64 row
    pointers, int32 columns), assembled from the blocks' CSR arrays."""
    parts = [_csr_arrays(a) for a in As]
    n = sum(len(rp) - 1 for rp, _, _ in parts)
    nnz = sum(int(rp[-1]) for rp, _, _ in parts)
    rp = np.zeros(n + 1, np.int64)
    ci = np.empty(nnz, np.int32)
    v = np.empty(nnz, np.float64)
    r0 = z0 = 0
    for prp, pci, pv in parts:
        nb, zb = len(prp) - 1, int(prp[-1])
        rp[r0 + 1:r0 + nb + 1] = prp[1:] + z0
        ci[z0:z0 + zb] = pci[:zb] + r0
        v[z0:z0 + zb] = pv[:zb]
        r0 += nb
        z0 += zb
    return sp.csr_matrix((v, ci, rp), shape=(n, n))


def read_matrix_market(path: str) -> sp.csr_matrix:
    """readMatrixMarket (src/io/matrix_market.cpp:48-97) through the C ABI."""
    n = C.c_int64(0)
    nnz = C.c_int64(0)
    _lib.check(_lib.lib().amls_mm_read(str(path).encode(), C.byref(n), C.byref(nnz), None, None, None))
    rp = np.zeros(n.value + 1, np.int64)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    v = np.zeros(max(nnz.value, 1), np.float64)
    _lib.check(_lib.lib().amls_mm_read(str(path).encode(), C.byref(n), C.byref(nnz), _lib.ptr(rp),
                                       _lib.ptr(ci), _lib.ptr(v)))
    return sp.csr_matrix((v[:nnz.value], ci[:nnz.value], rp), shape=(n.value, n.value))


def write_matrix_market(path: str, A) -> None:
    """writeMatrixMarket (src/io/matrix_market.cpp:99-115): lower triangle,
    real symmetric."""
    rp, ci, v = _csr_arrays(A)
    _lib.check(_lib.lib().amls_mm_write(str(path).encode(), A.shape[0], _lib.ptr(rp), _lib.ptr(ci),
                                        _lib.ptr(v)))


def element_pattern(n: int, dofmap: np.ndarray):
    """CSR pattern (rowptr, col) of an element mesh (amls_element_pattern)."""
    dm = np.ascontiguousarray(dofmap, dtype=np.int64)
    nnz = C.c_int64(0)
    _lib.check(_lib.lib().amls_element_pattern(int(n), dm.shape[0], dm.shape[1], _lib.ptr(dm), C.byref(nnz),
                                               None, None))
    rp = np.zeros(n + 1, np.int64)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    _lib.check(_lib.lib().amls_element_pattern(int(n), dm.shape[0], dm.shape[1], _lib.ptr(dm), C.byref(nnz),
                                               _lib.ptr(rp), _lib.ptr(ci)))
    return rp, ci[:nnz.value]


def recursive_bisection(K, M, nLevels: int, leafSize: int):
    """Partition of |K| + |M|: returns (perm, tree arrays dict)."""
    kp, kc, _ = _csr_arrays(K)
    mp, mc, _ = _csr_arrays(M)
    n = K.shape[0]
    perm = np.zeros(n, np.int64)
    nn = C.c_int64(0)
    parent = np.zeros(n, np.int64)
    role = np.zeros(n, np.int32)
    left = np.zeros(n, np.int64)
    right = np.zeros(n, np.int64)
    idx_ptr = np.zeros(n + 1, np.int64)
    idx = np.zeros(n, np.int64)
    _lib.check(_lib.lib().amls_partition(n, kp, kc, mp, mc, int(nLevels), int(leafSize), perm,
                                         C.byref(nn), parent, role, left, right, idx_ptr, idx))
    N = nn.value
    return perm, dict(parent=parent[:N].copy(), role=role[:N].copy(), left=left[:N].copy(),
                      right=right[:N].copy(), idx_ptr=idx_ptr[:N + 1].copy(), idx=idx.copy())


class AmlsSolver:
    """One GPU handle; ``solve`` is the drop-in for AmlsSolver::solve."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _lib.check(_lib.lib().amls_create(int(device), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            _lib.lib().amls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, K, M, opt: AmlsOptions) -> Solution:
        kp, kc, kv = _csr_arrays(K)
        mp, mc, mv = _csr_arrays(M)
        n = K.shape[0]
        nev = max(0, min(int(opt.nev), n))
        theta = np.zeros(max(nev, 1), np.float64)
        # every element of Z is written by the call (columns beyond the
        # values found are zero); Z.T is the n x nev column-major result
        Z = np.empty((nev, n), np.float64) if opt.recoverVectors and nev > 0 else None
        p = C.c_int64(0)
        timing = np.zeros(_lib.T_SLOTS, np.float64)
        o = opt.to_c()
        _lib.check(_lib.lib().amls_solve(self._h, n, _lib.ptr(kp), _lib.ptr(kc), _lib.ptr(kv),
                                         _lib.ptr(mp), _lib.ptr(mc), _lib.ptr(mv), C.byref(o),
                                         _lib.ptr(theta), _lib.ptr(Z), C.byref(p),
                                         _lib.ptr(timing)))
        self._last_nev = nev
        return Solution(theta[:nev].copy(), None if Z is None else Z.T, int(p.value),
                        dict(zip(_lib.TIMING_KEYS, timing.tolist())), self.info())

    # ---- batch of independent pencils (one launch sequence) ----
    def solve_batch(self, Ks, Ms, opt: AmlsOptions):
        """Each pencil (Ks[b], Ms[b]) solved as by ``solve`` (its own
        partition and two-pass truncation), all of them level-batched on the
        GPU.  Returns a list of Solution (theta, Z per pencil; p and timing of
        the whole batch)."""
        K = _block_diag(Ks)
        M = _block_diag(Ms)
        off = np.zeros(len(Ks) + 1, np.int64)
        off[1:] = np.cumsum([k.shape[0] for k in Ks])
        kp, kc, kv = _csr_arrays(K)
        mp, mc, mv = _csr_arrays(M)
        n = int(off[-1])
        nev = max(1, min(int(opt.nev), n))
        B = len(Ks)
        theta = np.zeros(B * nev, np.float64)
        m = np.zeros(B, np.int64)
        Z = np.zeros((nev, n), np.float64) if opt.recoverVectors else None
        timing = np.zeros(_lib.T_SLOTS, np.float64)
        o = opt.to_c()
        _lib.check(_lib.lib().amls_solve_batch(self._h, B, _lib.ptr(off), _lib.ptr(kp), _lib.ptr(kc),
                                               _lib.ptr(kv), _lib.ptr(mp), _lib.ptr(mc), _lib.ptr(mv),
                                               C.byref(o), _lib.ptr(theta), _lib.ptr(m), _lib.ptr(Z),
                                               _lib.ptr(timing)))
        info = self.info()
        tim = dict(zip(_lib.TIMING_KEYS, timing.tolist()))
        out = []
        for b in range(B):
            mb = int(m[b])
            Zb = None if Z is None else Z[:mb, off[b]:off[b + 1]].T.copy()
            out.append(Solution(theta[b * nev:b * nev + mb].copy(), Zb, -1, tim, info))
        return out

    def analyze_batch(self, Ks, Ms, opt: AmlsOptions):
        """Pattern analysis of a batch; returns the block-diagonal (K, M) whose
        .data arrays are the value order of solve_values_batch."""
        K = _block_diag(Ks)
        M = _block_diag(Ms)
        off = np.zeros(len(Ks) + 1, np.int64)
        off[1:] = np.cumsum([k.shape[0] for k in Ks])
        kp, kc, _ = _csr_arrays(K)
        mp, mc, _ = _csr_arrays(M)
        o = opt.to_c()
        _lib.check(_lib.lib().amls_analyze_batch(self._h, len(Ks), _lib.ptr(off), _lib.ptr(kp),
                                                 _lib.ptr(kc), _lib.ptr(mp), _lib.ptr(mc), C.byref(o)))
        self._batch_off = off
        return K, M

    def solve_values_batch(self, k_val_ptr: int, m_val_ptr: int, values_on_device: bool,
                           theta_ptr: int, m_ptr: int, z_ptr: int | None,
                           outputs_on_device: bool) -> dict:
        timing = np.zeros(_lib.T_SLOTS, np.float64)
        _lib.check(_lib.lib().amls_solve_values_batch(
            self._h, C.c_void_p(k_val_ptr), C.c_void_p(m_val_ptr), 1 if values_on_device else 0,
            C.c_void_p(theta_ptr), C.c_void_p(m_ptr), None if z_ptr is None else C.c_void_p(z_ptr),
            1 if outputs_on_device else 0, _lib.ptr(timing)))
        return dict(zip(_lib.TIMING_KEYS, timing.tolist()))

    # ---- split form: analysis once, numeric solves on resident values ----
    def analyze(self, K, M, opt: AmlsOptions) -> None:
        kp, kc, _ = _csr_arrays(K)
        mp, mc, _ = _csr_arrays(M)
        self._n = K.shape[0]
        self._nev = max(0, min(int(opt.nev), self._n))
        o = opt.to_c()
        _lib.check(_lib.lib().amls_analyze(self._h, self._n, _lib.ptr(kp), _lib.ptr(kc),
                                           _lib.ptr(mp), _lib.ptr(mc), C.byref(o)))

    def solve_values(self, k_val_ptr: int, m_val_ptr: int, values_on_device: bool,
                     theta_ptr: int, z_ptr: int | None, outputs_on_device: bool) -> dict:
        """Numeric solve on the analysed pattern; pointers are raw addresses
        (device addresses when the *_on_device flags are set)."""
        p = C.c_int64(0)
        timing = np.zeros(_lib.T_SLOTS, np.float64)
        _lib.check(_lib.lib().amls_solve_values(
            self._h, C.c_void_p(k_val_ptr), C.c_void_p(m_val_ptr), 1 if values_on_device else 0,
            C.c_void_p(theta_ptr), None if z_ptr is None else C.c_void_p(z_ptr),
            1 if outputs_on_device else 0, C.byref(p), _lib.ptr(timing)))
        out = dict(zip(_lib.TIMING_KEYS, timing.tolist()))
        out["p"] = int(p.value)
        return out

    # ---- stage by stage (the reference's pipeline seams) ----
    def eliminate(self, K, M) -> None:
        """GaussianElimination::run on the analysed pattern with these values."""
        _, _, kv = _csr_arrays(K)
        _, _, mv = _csr_arrays(M)
        _lib.check(_lib.lib().amls_eliminate(self._h, _lib.ptr(kv), _lib.ptr(mv), 0))

    def condense(self, mode: str, k: int = 0, lambda_cut: float = 0.0) -> int:
        """SubspaceCondensation::run with FixedCountTruncation(k) ("fixed") or
        ThresholdTruncation(lambda_cut) ("threshold"); returns p."""
        p = C.c_int64(0)
        _lib.check(_lib.lib().amls_condense(self._h, 0 if mode == "fixed" else 1, int(k), float(lambda_cut),
                                            C.byref(p)))
        self._p = p.value
        return p.value

    def pass_modes(self):
        """(kept count per tree node, local eigenvalues mu in node-id order)."""
        t = self.tree()
        k = np.zeros(len(t["parent"]), np.int32)
        mu = np.zeros(max(self._p, 1))
        _lib.check(_lib.lib().amls_pass_modes(self._h, _lib.ptr(k), _lib.ptr(mu)))
        return k, mu[:self._p]

    def reduced_eig(self, want: int, vectors: bool = True) -> np.ndarray:
        theta = np.zeros(max(int(want), 1))
        m = C.c_int64(0)
        _lib.check(_lib.lib().amls_reduced_eig(self._h, int(want), 1 if vectors else 0, _lib.ptr(theta),
                                               C.byref(m)))
        self._m = m.value
        return theta[:m.value].copy()

    def backtransform(self) -> np.ndarray:
        n = self.info()["n"]
        Z = np.zeros((self._m, n))
        m = C.c_int64(0)
        _lib.check(_lib.lib().amls_backtransform(self._h, _lib.ptr(Z), 0, C.byref(m)))
        return Z[:m.value].T.copy()

    def refine(self, nev: int):
        n = self.info()["n"]
        theta = np.zeros(int(nev))
        Z = np.zeros((int(nev), n))
        it = C.c_int64(0)
        _lib.check(_lib.lib().amls_refine(self._h, int(nev), _lib.ptr(theta), _lib.ptr(Z), 0, C.byref(it)))
        self._last_nev = int(nev)
        return theta, Z.T.copy(), int(it.value)

    def tree(self) -> dict:
        nn = C.c_int64(0)
        _lib.check(_lib.lib().amls_tree(self._h, C.byref(nn), None, None, None))
        N = nn.value
        parent = np.zeros(N, np.int64)
        size = np.zeros(N, np.int64)
        level = np.zeros(N, np.int32)
        _lib.check(_lib.lib().amls_tree(self._h, C.byref(nn), _lib.ptr(parent), _lib.ptr(size), _lib.ptr(level)))
        return dict(parent=parent, size=size, level=level)

    def assemble_hex(self, pencil, rowptr, col, on_device: bool = False, k_ptr: int = 0, m_ptr: int = 0):
        """K and M values of a hex pencil's mesh assembled on the GPU in the
        pattern (rowptr, col): host arrays returned, or written to the device
        pointers k_ptr / m_ptr with on_device."""
        coords = np.ascontiguousarray(pencil.coords, dtype=np.float64)
        en = np.ascontiguousarray(pencil.enodes, dtype=np.int64)
        dm = np.ascontiguousarray(pencil.dofmap, dtype=np.int64)
        E = np.ascontiguousarray(pencil.E, dtype=np.float64)
        rho = np.ascontiguousarray(pencil.rho, dtype=np.float64)
        rp = np.ascontiguousarray(rowptr, dtype=np.int64)
        ci = np.ascontiguousarray(col, dtype=np.int32)
        n = rp.size - 1
        if on_device:
            kv, mv = C.c_void_p(k_ptr), C.c_void_p(m_ptr)
        else:
            kh = np.zeros(max(ci.size, 1))
            mh = np.zeros(max(ci.size, 1))
            kv, mv = _lib.ptr(kh), _lib.ptr(mh)
        _lib.check(_lib.lib().amls_hex_assemble(self._h, int(pencil.order), en.shape[0], coords.shape[0],
                                                _lib.ptr(coords), _lib.ptr(en), _lib.ptr(dm), _lib.ptr(E),
                                                _lib.ptr(rho), float(pencil.nu), n, _lib.ptr(rp), _lib.ptr(ci),
                                                kv, mv, 1 if on_device else 0))
        if on_device:
            return None
        return (sp.csr_matrix((kh[:ci.size], ci, rp), shape=(n, n)),
                sp.csr_matrix((mh[:ci.size], ci, rp), shape=(n, n)))

    def sensitivities(self, pencil, weights=None, per_mode: bool = False, gap_tol: float = 1e-6,
                      elem_type=None):
        """Per-element eigenvalue sensitivities of the last solve's eigenpairs
        for an element pencil (K = sum E_e Kbar_t(e), M = sum rho_e Mbar_t(e)).
        ``pencil.Kbar``/``pencil.Mbar`` are one element pair (nd x nd) or a
        stack (ntypes x nd x nd) indexed by ``elem_type`` (nelem ints).
        Returns dict(gE, gRho, simple[, dE, dRho]) with gE/gRho the gradient of
        sum_k w_k lambda_k over simple modes (zeros without weights) and
        dE/dRho of shape (nelem, nev) when per_mode."""
        dm = np.ascontiguousarray(pencil.dofmap, dtype=np.int64)
        nelem, nd = dm.shape
        Kbar = np.asarray(pencil.Kbar, dtype=np.float64)
        Mbar = np.asarray(pencil.Mbar, dtype=np.float64)
        if Kbar.ndim == 2:
            Kbar, Mbar = Kbar[None], Mbar[None]
        ntypes = Kbar.shape[0]
        Kb = np.ascontiguousarray(Kbar.transpose(0, 2, 1)).ravel()      # column-major per type
        Mb = np.ascontiguousarray(Mbar.transpose(0, 2, 1)).ravel()
        et = None if elem_type is None else np.ascontiguousarray(elem_type, dtype=np.int32)
        nev = self._last_nev
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        gE = np.zeros(nelem)
        gR = np.zeros(nelem)
        simple = np.zeros(nev, np.int32)
        dE = np.zeros((nev, nelem)) if per_mode else None
        dR = np.zeros((nev, nelem)) if per_mode else None
        _lib.check(_lib.lib().amls_sensitivities(
            self._h, nelem, nd, _lib.ptr(dm), int(ntypes), _lib.ptr(et), _lib.ptr(Kb), _lib.ptr(Mb),
            _lib.ptr(w),
            float(gap_tol), _lib.ptr(gE), _lib.ptr(gR), _lib.ptr(dE), _lib.ptr(dR),
            _lib.ptr(simple)))
        out = dict(gE=gE, gRho=gR, simple=simple.astype(bool))
        if per_mode:
            out["dE"] = dE.T.copy()
            out["dRho"] = dR.T.copy()
        return out

    def set_profiling(self, on: bool) -> None:
        _lib.check(_lib.lib().amls_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        ms = np.zeros(len(_lib.PROF_CATS), np.float64)
        cnt = np.zeros(len(_lib.PROF_CATS), np.int64)
        _lib.check(_lib.lib().amls_kernel_times(self._h, _lib.ptr(ms), _lib.ptr(cnt)))
        return {k: (float(a), int(b)) for k, a, b in zip(_lib.PROF_CATS, ms, cnt)}

    def category_work(self) -> dict:
        """Algorithmic (flops, bytes) of the last solve per kernel category."""
        f = np.zeros(len(_lib.PROF_CATS), np.float64)
        b = np.zeros(len(_lib.PROF_CATS), np.float64)
        _lib.check(_lib.lib().amls_category_work(self._h, _lib.ptr(f), _lib.ptr(b)))
        return {k: (float(x), float(y)) for k, x, y in zip(_lib.PROF_CATS, f, b)}

    def info(self) -> dict:
        buf = np.zeros(_lib.INFO_SLOTS, np.int64)
        _lib.check(_lib.lib().amls_info(self._h, _lib.ptr(buf)))
        keys = ["tree_nodes", "levels", "p_passA", "p", "front_doubles", "device_bytes",
                "launches", "refine_iters", "refine_nq", "n", "sil_nodes", "sil_served"]
        return {k: int(v) for k, v in zip(keys, buf)}

    def permutation(self) -> np.ndarray:
        """perm[new] = old of the last analysis on this handle."""
        out = np.zeros(self.info()["n"], np.int64)
        _lib.check(_lib.lib().amls_permutation(self._h, _lib.ptr(out)))
        return out

    def work(self) -> dict:
        buf = np.zeros(_lib.WORK_SLOTS, np.float64)
        _lib.check(_lib.lib().amls_work(self._h, _lib.ptr(buf)))
        keys = ["flops_elim", "bytes_elim", "flops_cond", "bytes_cond", "flops_reduced",
                "bytes_reduced", "flops_back", "bytes_back"]
        return dict(zip(keys, buf.tolist()))


def sygvx_batched(solver: AmlsSolver, Ks, Ms, mode: str = "index", il: int = 1, iu: int = 1,
                  lo: float = -1e300, hi: float = 0.0):
    """Lowest eigenpairs of each dense pencil (K_b, M_b) on the GPU
    (dsygvx semantics, dense_eigensolver.cpp:44-133).  Returns lists (w_b, V_b)."""
    B = len(Ks)
    n = np.array([k.shape[0] for k in Ks], np.int64)
    mat_off = np.zeros(B, np.int64)
    mat_off[1:] = np.cumsum(n * n)[:-1]
    Kf = np.concatenate([np.asfortranarray(k).ravel(order="F") for k in Ks]).astype(np.float64)
    Mf = np.concatenate([np.asfortranarray(m).ravel(order="F") for m in Ms]).astype(np.float64)
    cap = n.copy() if mode != "index" else np.minimum(n, iu - il + 1)
    w_off = np.zeros(B, np.int64)
    w_off[1:] = np.cumsum(cap)[:-1]
    v_off = np.zeros(B, np.int64)
    v_off[1:] = np.cumsum(n * cap)[:-1]
    w = np.zeros(max(int(cap.sum()), 1))
    V = np.zeros(max(int((n * cap).sum()), 1))
    m = np.zeros(B, np.int64)
    _lib.check(_lib.lib().amls_sygvx_batched(
        solver._h, B, _lib.ptr(n), _lib.ptr(mat_off), _lib.ptr(Kf), _lib.ptr(Mf),
        0 if mode == "index" else 1, int(il), int(iu), float(lo), float(hi), _lib.ptr(cap),
        _lib.ptr(w_off), _lib.ptr(w), _lib.ptr(v_off), _lib.ptr(V), _lib.ptr(m)))
    out = []
    for b in range(B):
        mb, nb = int(m[b]), int(n[b])
        wb = w[w_off[b]:w_off[b] + mb].copy()
        Vb = V[v_off[b]:v_off[b] + nb * mb].reshape(mb, nb).T.copy()
        out.append((wb, Vb))
    return out
