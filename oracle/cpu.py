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
METIS_SRC = os.path.join(HERE, "metis_seq.cpp")
METIS_LIB = os.path.join(HERE, "libmetis_seq.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
METIS_A = os.path.join(CUDA, "targets", "x86_64-linux", "lib", "libmetis_static.a")


def build() -> str:
    """Both oracle libraries: the C++ restatement of the AMLS algorithm and
    the sequential restatement of the reference's nested dissection (linked
    with the METIS library of the CUDA toolkit)."""
    for src, lib, extra in ((SRC, LIB, ["-ldl", "-lpthread"]), (METIS_SRC, METIS_LIB, [METIS_A, "-lm"])):
        if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-Wall", src, "-o", lib, *extra]
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


def sequential_partition(K, M, n_levels: int, leaf_size: int):
    """The reference's MetisPartitioner::recursiveBisection restated
    sequentially (oracle/metis_seq.cpp, with its METIS_PartGraphRecursive
    call): (perm, tree arrays) as amls_b200.solver.recursive_bisection."""
    build()
    L = C.CDLL(METIS_LIB)
    P = C.c_void_p
    L.metis_seq_partition.argtypes = [C.c_int64, P, P, P, P, C.c_int, C.c_int64, P, P, P, P, P, P, P, P]
    K = sp.csr_matrix(K)
    M = sp.csr_matrix(M)
    K.sort_indices()
    M.sort_indices()
    n = K.shape[0]
    kp = np.ascontiguousarray(K.indptr, np.int64)
    kc = np.ascontiguousarray(K.indices, np.int32)
    mp = np.ascontiguousarray(M.indptr, np.int64)
    mc = np.ascontiguousarray(M.indices, np.int32)
    perm = np.zeros(n, np.int64)
    nn = C.c_int64(0)
    parent = np.zeros(n, np.int64)
    role = np.zeros(n, np.int32)
    left = np.zeros(n, np.int64)
    right = np.zeros(n, np.int64)
    ip = np.zeros(n + 1, np.int64)
    ix = np.zeros(n, np.int64)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)   # noqa: E731
    rc = L.metis_seq_partition(n, ptr(kp), ptr(kc), ptr(mp), ptr(mc), int(n_levels), int(leaf_size), ptr(perm),
                               C.byref(nn), ptr(parent), ptr(role), ptr(left), ptr(right), ptr(ip), ptr(ix))
    if rc != 0:
        raise RuntimeError("METIS failed")
    N = nn.value
    return perm, dict(parent=parent[:N].copy(), role=role[:N].copy(), left=left[:N].copy(),
                      right=right[:N].copy(), idx_ptr=ip[:N + 1].copy(), idx=ix.copy())
