"""Algorithmic work model of the reference AMLS algorithm (test
infrastructure: used only to scale the CPU baseline's bounded sample).

For every tree node i with n_i own DOFs and s_i coupled ancestor DOFs after
fill (the reference's symbolic fill, src/amls/gaussian_elimination.cpp:
221-270, taken over the union pattern of K and M), the reference spends
  factor          n_i^3 / 3                          (factorNode_ :458-508)
  X, Y solves     2 * 2 n_i^2 s_i                    (solveXYAnc_ :510-598)
  WX              2 n_i^2 s_i + 2 n_i^2 s_i          (makeWX_ :653-676)
  K Schur         2 s_i^2 n_i                        (schurK* :678-715)
  M congruence    3 * 2 s_i^2 n_i                    (cong* :717-781)
  local eigs      2 passes x 3 n_i^3 (dsygvx: potrf + sygst + sytrd)
plus 2 passes x 4/3 p^3 for the reduced problems.  The model is used as a
ratio (full workload / sample), so its constant factors cancel to first
order.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .tree import Tree


def fill_sets(K: sp.csr_matrix, M: sp.csr_matrix, tree: Tree):
    """S_i (as sorted arrays of permuted indices) for every node."""
    perm = tree.perm()
    n = len(perm)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    order = tree.post_order()
    off, size = {}, {}
    acc = 0
    for i in order:
        off[i] = acc
        size[i] = len(tree.indices[i])
        acc += size[i]
    owner = np.empty(n, dtype=np.int64)
    for i in order:
        owner[off[i]:off[i] + size[i]] = i
    A = sp.csr_matrix(K + M)
    push = {i: [] for i in order}
    S = {}
    for i in order:
        rows_old = perm[off[i]:off[i] + size[i]]
        sub = A[rows_old, :]
        cols = inv[sub.indices]
        anc = set(tree.ancestors(i))
        mine = cols[np.isin(owner[cols], list(anc))] if anc else np.zeros(0, np.int64)
        allc = np.unique(np.concatenate([mine] + [np.asarray(x, np.int64) for x in push[i]]))
        S[i] = allc
        if allc.size:
            a0 = owner[allc[0]]
            end0 = off[a0] + size[a0]
            push[a0].append(allc[allc >= end0])
    return S, size


def amls_work(K, M, tree: Tree, p_final: int, p_a: int) -> float:
    S, size = fill_sets(K, M, tree)
    w = 0.0
    for i, s_arr in S.items():
        n_i = float(size[i])
        s_i = float(len(s_arr))
        w += n_i ** 3 / 3 + 4 * n_i ** 2 * s_i + 4 * n_i ** 2 * s_i + 8 * s_i ** 2 * n_i
        w += 6 * n_i ** 3
    w += 4.0 / 3.0 * (float(p_final) ** 3 + float(p_a) ** 3)
    return w
