"""Shared helpers of the test-suite: partition + oracle runs on a pencil."""
from __future__ import annotations

import numpy as np

from amls_b200 import cases, solver as S
from oracle import amls_ref as R
from oracle.tree import Tree


def partition(p: cases.Pencil, nLevels: int, leafSize: int):
    perm, t = S.recursive_bisection(p.K, p.M, nLevels, leafSize)
    return perm, Tree.from_arrays(**t)


def oracle_solve(p: cases.Pencil, opt: R.OptionsRef):
    _, tree = partition(p, opt.nLevels, opt.leafSize)
    return R.amls_solve_ref(p.K, p.M, tree, opt)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def residuals(K, M, theta, Z):
    """||K z - theta M z|| / (||K|| ||z||) per column (||K|| = max abs row sum)."""
    KZ = K @ Z
    MZ = M @ Z
    R_ = KZ - MZ * theta[None, :]
    knorm = abs(K).sum(axis=1).max()
    return np.linalg.norm(R_, axis=0) / (knorm * np.linalg.norm(Z, axis=0))
