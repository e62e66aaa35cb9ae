"""Separator tree as plain Python data (test infrastructure: the oracle).

Mirrors the reference's SeparatorTree (src/amls/separator_tree.cpp:26-107):
node ids in creation order, children [left, right], post-order = children
then self, ancestors = parent .. root, "level" = height from the leaves
(src/amls/gaussian_elimination.cpp:134-148).
"""
from __future__ import annotations

import dataclasses

import numpy as np

LEAF, SEPARATOR, ROOT = 0, 1, 2


@dataclasses.dataclass
class Tree:
    parent: list[int]
    role: list[int]
    children: list[list[int]]
    indices: list[np.ndarray]          # original indices per node

    @property
    def n_nodes(self) -> int:
        return len(self.parent)

    def root(self) -> int:
        return self.parent.index(-1)

    def post_order(self) -> list[int]:
        out: list[int] = []
        stack = [(self.root(), False)]
        while stack:
            nd, done = stack.pop()
            if done:
                out.append(nd)
                continue
            stack.append((nd, True))
            for c in reversed(self.children[nd]):
                stack.append((c, False))
        return out

    def ancestors(self, i: int) -> list[int]:
        out = []
        p = self.parent[i]
        while p != -1:
            out.append(p)
            p = self.parent[p]
        return out

    def levels(self) -> list[int]:
        lev = [0] * self.n_nodes
        for i in self.post_order():
            if self.children[i]:
                lev[i] = max(lev[c] + 1 for c in self.children[i])
        return lev

    def is_leaf(self, i: int) -> bool:
        return self.role[i] == LEAF

    def perm(self) -> np.ndarray:
        return np.concatenate([self.indices[i] for i in self.post_order()]).astype(np.int64)

    @staticmethod
    def from_arrays(parent, role, left, right, idx_ptr, idx) -> "Tree":
        n_nodes = len(parent)
        children = [[] if left[i] < 0 else [int(left[i]), int(right[i])] for i in range(n_nodes)]
        indices = [np.asarray(idx[idx_ptr[i]:idx_ptr[i + 1]], dtype=np.int64) for i in range(n_nodes)]
        return Tree([int(p) for p in parent], [int(r) for r in role], children, indices)
