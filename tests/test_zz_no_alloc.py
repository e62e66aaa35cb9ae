"""The allocation-free eigensolver entry point (amls_sygvx_lowest_noalloc).

It exists for callers that cannot allocate device memory (hosts whose own
pool owns every device allocation, loops that must not enter the
allocator): inputs and outputs are the caller's device buffers and all
scratch is a fixed device array inside the library.  Its results must equal
LAPACK dsygvx (index range [1, k], itype 1, uplo 'L' - the reference's
LapackDenseEigensolver::solveIndex) and the allocating batched entry point
(amls_sygvx_batched) on the same pencils, on two calls in a row (the second
call reuses the scratch the first one left behind).  Orders that are not
multiples of the 32-wide tiles exercise the partial edge tiles; an M that is
not positive definite must return AMLS_ERR_NOT_SPD and leave the entry point
usable.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from amls_b200 import _lib, sygvx_batched
from oracle import amls_ref as R

pytestmark = pytest.mark.gpu

# (n, k, seed): k = 1, k = n, n = 1, odd orders with partial 32-wide tiles,
# and the largest accepted order
CASES = [(96, 10, 1), (_lib.NOALLOC_MAX_N, 17, 2), (1, 1, 3), (40, 40, 4), (77, 1, 5),
         (127, 40, 6)]


def _pencil(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    return A @ A.T + n * np.eye(n), B @ B.T / n + np.eye(n)


def _noalloc(K, M, k):
    import torch
    n = K.shape[0]
    dK = torch.from_numpy(np.asfortranarray(K).ravel(order="F").copy()).cuda()
    dM = torch.from_numpy(np.asfortranarray(M).ravel(order="F").copy()).cuda()
    dw = torch.zeros(k, dtype=torch.float64, device="cuda")
    dV = torch.zeros(n * k, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    m = C.c_int64(-1)
    rc = _lib.lib().amls_sygvx_lowest_noalloc(n, dK.data_ptr(), dM.data_ptr(), k, dw.data_ptr(),
                                              dV.data_ptr(), C.byref(m), None)
    torch.cuda.synchronize()
    return rc, m.value, dw.cpu().numpy(), dV.cpu().numpy().reshape(k, n).T


def _check(K, M, k, w, V, wb, Vb):
    wr, Vr = R.LapackDense.solve_index(K, M, 1, k)
    assert np.max(np.abs(w - wr) / np.abs(wr)) < 1e-12
    assert np.max(np.abs(w - wb) / np.abs(wb)) < 1e-12
    for ref in (Vb, Vr):
        sign = np.sign(np.sum(V * (M @ ref), axis=0))
        assert np.max(np.abs(V * sign - ref)) < 1e-10 * np.max(np.abs(ref))
    assert np.allclose(V.T @ M @ V, np.eye(k), atol=1e-10)


@pytest.mark.parametrize("n,k,seed", CASES)
def test_noalloc_matches_lapack_and_allocating_entry_point_two_calls(solver, n, k, seed):
    K, M = _pencil(n, seed)
    (wb, Vb), = sygvx_batched(solver, [K], [M], mode="index", il=1, iu=k)
    for _ in range(2):
        rc, m, w, V = _noalloc(K, M, k)
        assert rc == _lib.AMLS_OK, _lib.lib().amls_last_error()
        assert m == k
        _check(K, M, k, w, V, wb, Vb)


def test_noalloc_reports_indefinite_m_and_stays_usable(solver):
    n, k = 70, 5
    K, M = _pencil(n, 7)
    Mbad = M.copy()
    Mbad[10, 10] = -5.0
    rc, _, _, _ = _noalloc(K, Mbad, k)
    assert rc == _lib.AMLS_ERR_NOT_SPD
    (wb, Vb), = sygvx_batched(solver, [K], [M], mode="index", il=1, iu=k)
    rc, m, w, V = _noalloc(K, M, k)
    assert rc == _lib.AMLS_OK and m == k
    _check(K, M, k, w, V, wb, Vb)


def test_noalloc_rejects_sizes_beyond_the_limit():
    m = C.c_int64(0)
    rc = _lib.lib().amls_sygvx_lowest_noalloc(_lib.NOALLOC_MAX_N + 1, 1, 1, 1, 1, 1, C.byref(m),
                                              None)
    assert rc == _lib.AMLS_ERR_INVALID_ARGUMENT
    rc = _lib.lib().amls_sygvx_lowest_noalloc(10, 1, 1, 11, 1, 1, C.byref(m), None)
    assert rc == _lib.AMLS_ERR_INVALID_ARGUMENT
