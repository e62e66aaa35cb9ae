"""The C++ restatement of the reference algorithm (oracle/amls_cpu.cpp):
build recipe and ctypes binding.  Test infrastructure and the timed CPU
baseline - the product never loads it.

``build()`` compiles amls_cpu.cpp with g++ into oracle/libamls_cpu.so;
``solve(K, M, tree, ...)`` runs it on a given partition tree (the tree
arrays of the host partition: parent, left, right, idx_ptr, idx), with the
LAPACK/BLAS of the OpenBLAS that scipy ships, single-threaded per call and
parallel over the nodes of a tree level as the reference is.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "amls_cpu.cpp")
LIB = os.path.join(HERE, "libamls_cpu.so")


def build() -> str:
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-Wall", SRC, "-o", LIB, "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed: {' '.join(cmd)}\n{r.stderr}")
    return LIB


def blas_path() -> str:
    import scipy
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(d, "libscipy_openblas-*.so")))
    if not cands:
        raise RuntimeError("scipy's OpenBLAS (LP64) not found")
    return cands[0]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.amls_cpu_solve.argtypes = [C.c_char_p, C.c_int, C.c_int64, P, P, P, P, P, P, C.c_int, P, P, P, P, P,
                                     C.c_int, C.c_double, C.c_int, C.c_int, P, P, P, P, P, C.c_char_p, C.c_int]
        _lib = L
    return _lib


def solve(K, M, tree: dict, nev: int, eta: float = 2.0, fixed_keep: int = 0, vectors: bool = True,
          threads: int | None = None, rerun_elimination: bool = True):
    """AmlsSolver::solve (src/amls/solver.cpp:100-319) on the given tree.
    Returns (theta, Z or None, p, p of pass A, timing dict)."""
    K = sp.csr_matrix(K)
    M = sp.csr_matrix(M)
    K.sort_indices()
    M.sort_indices()
    n = K.shape[0]
    nev = min(nev, n)
    threads = threads or (os.cpu_count() or 1)
    arr = lambda a, t: np.ascontiguousarray(a, dtype=t)   # noqa: E731
    kp, kc, kv = arr(K.indptr, np.int64), arr(K.indices, np.int32), arr(K.data, np.float64)
    mp, mc, mv = arr(M.indptr, np.int64), arr(M.indices, np.int32), arr(M.data, np.float64)
    par, le, ri = (arr(tree[k], np.int64) for k in ("parent", "left", "right"))
    ip, ix = arr(tree["idx_ptr"], np.int64), arr(tree["idx"], np.int64)
    theta = np.zeros(nev)
    Z = np.zeros((nev, n)) if vectors else None
    p = C.c_int64(0)
    pa = C.c_int64(0)
    tm = np.zeros(6)
    err = C.create_string_buffer(512)
    ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)   # noqa: E731
    rc = lib().amls_cpu_solve(blas_path().encode(), int(threads), n, ptr(kp), ptr(kc), ptr(kv), ptr(mp), ptr(mc),
                              ptr(mv), len(par), ptr(par), ptr(le), ptr(ri), ptr(ip), ptr(ix), int(nev), float(eta),
                              int(fixed_keep), 1 if rerun_elimination else 0, ptr(theta), ptr(Z), C.byref(p),
                              C.byref(pa), ptr(tm), err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    keys = ["permutation", "elimination", "condensation", "reduced", "backtransform", "total"]
    return theta, (None if Z is None else Z.T.copy()), int(p.value), int(pa.value), dict(zip(keys, tm.tolist()))
