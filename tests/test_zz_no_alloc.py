"""The allocation-free eigensolver entry point (amls_sygvx_lowest_noalloc).

It exists for callers that cannot allocate device memory (graph capture,
hosts whose pool owns all allocations, allocator-free loops): inputs and
outputs are the caller's device buffers and all scratch is a fixed device
array inside the library.  Its results must equal those of the allocating
batched entry point (amls_sygvx_batched) on the same pencils, on two calls in
a row (the second call reuses the scratch the first one left behind).

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from amls_b200 import _lib, sygvx_batched

pytestmark = pytest.mark.gpu


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


def test_noalloc_matches_allocating_entry_point_two_calls(solver):
    for n, k, seed in [(96, 10, 1), (_lib.NOALLOC_MAX_N, 17, 2)]:
        K, M = _pencil(n, seed)
        rc, m, w, V = _noalloc(K, M, k)
        assert rc == _lib.AMLS_OK, _lib.lib().amls_last_error()
        assert m == k
        (wb, Vb), = sygvx_batched(solver, [K], [M], mode="index", il=1, iu=k)
        assert np.max(np.abs(w - wb) / np.abs(wb)) < 1e-12
        sign = np.sign(np.sum(V * Vb, axis=0))
        assert np.max(np.abs(V * sign - Vb)) < 1e-10 * np.max(np.abs(Vb))
        assert np.allclose(V.T @ M @ V, np.eye(k), atol=1e-10)


def test_noalloc_rejects_sizes_beyond_the_limit():
    m = C.c_int64(0)
    rc = _lib.lib().amls_sygvx_lowest_noalloc(_lib.NOALLOC_MAX_N + 1, 1, 1, 1, 1, 1, C.byref(m),
                                              None)
    assert rc == _lib.AMLS_ERR_INVALID_ARGUMENT
    rc = _lib.lib().amls_sygvx_lowest_noalloc(10, 1, 1, 11, 1, 1, C.byref(m), None)
    assert rc == _lib.AMLS_ERR_INVALID_ARGUMENT
