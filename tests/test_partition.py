"""Host partitioner (METIS nested dissection) tests, no GPU needed.

Restates tests/unit/test_partition.cpp:16-101 of the reference: valid tree
with 2-8 leaves at 3 levels, perm[new] = old with post-order segments,
permuted diagonal blocks equal the original ones; plus determinism.
"""
import numpy as np
import pytest

from amls_b200 import cases, recursive_bisection
from oracle import amls_ref as R
from oracle.tree import LEAF, ROOT, Tree

from .helpers import partition


def test_tree_valid_three_levels():
    p = cases.grid_graph_2d(30, 30)
    perm, tree = partition(p, 3, 50)
    leaves = [i for i in range(tree.n_nodes) if tree.role[i] == LEAF]
    assert 2 <= len(leaves) <= 8
    assert tree.role[tree.root()] == ROOT
    allidx = np.sort(np.concatenate(tree.indices))
    assert np.array_equal(allidx, np.arange(p.n))
    for i in range(tree.n_nodes):
        for c in tree.children[i]:
            assert tree.parent[c] == i
        assert len(tree.children[i]) in (0, 2)


def test_perm_is_post_order_concatenation():
    p = cases.hex_pencil(5, 4, 4, 1, seed=0)
    perm, tree = partition(p, 3, 60)
    assert np.array_equal(perm, tree.perm())
    off = 0
    for i in tree.post_order():
        seg = perm[off:off + len(tree.indices[i])]
        assert np.array_equal(seg, tree.indices[i])
        off += len(seg)


def test_permuted_diag_blocks_equal_original():
    p = cases.grid_graph_2d(12, 12)
    perm, tree = partition(p, 2, 30)
    B = R.permute_symmetric(p.K, perm).toarray()
    A = p.K.toarray()
    off = 0
    for i in tree.post_order():
        idx = tree.indices[i]
        n = len(idx)
        assert np.abs(B[off:off + n, off:off + n] - A[np.ix_(idx, idx)]).max() < 1e-15
        off += n


def test_separators_disconnect_subtrees():
    """No matrix entry couples two different subtrees (vertex separators)."""
    p = cases.hex_pencil(6, 6, 6, 1, seed=1)
    perm, tree = partition(p, 4, 100)
    node_of = np.empty(p.n, dtype=np.int64)
    for i in range(tree.n_nodes):
        node_of[tree.indices[i]] = i
    anc = [set(tree.ancestors(i)) for i in range(tree.n_nodes)]
    rows = np.repeat(np.arange(p.n), np.diff(p.K.indptr))
    a, b = node_of[rows], node_of[p.K.indices]
    for x, y in set(zip(a.tolist(), b.tolist())):
        assert x == y or x in anc[y] or y in anc[x]


def test_partition_deterministic_and_leaf_rule():
    p = cases.hex_pencil(6, 5, 5, 1, seed=2)
    perm1, t1 = recursive_bisection(p.K, p.M, 3, 100)
    perm2, t2 = recursive_bisection(p.K, p.M, 3, 100)
    assert np.array_equal(perm1, perm2)
    for k in t1:
        assert np.array_equal(t1[k], t2[k])
    # stop rule m <= leafSize: a pencil smaller than leafSize is one leaf
    small = cases.path_graph(40)
    perm, t = recursive_bisection(small.K, small.M, 5, 100)
    assert len(t["parent"]) == 1 and np.array_equal(perm, np.arange(40))
    tree = Tree.from_arrays(**t)
    assert tree.role[0] == LEAF


@pytest.mark.parametrize("case", ["C1", "C2", "grid", "hexbox"])
def test_parallel_partition_equals_sequential_restatement(case):
    """The parallel partitioner (adjacency built per vertex in parallel, the
    unread METIS_PartGraphRecursive call dropped, concurrent subtrees in
    worker processes) returns the same permutation and tree as a literal
    sequential restatement of metis_partitioner.cpp that keeps every call
    (oracle/metis_seq.cpp)."""
    from amls_b200 import cases
    from amls_b200.solver import recursive_bisection
    from oracle import cpu
    p, L, leaf = {
        "C1": (cases.config_pencil("C1"), 4, 500),
        "C2": (cases.config_pencil("C2"), 6, 500),
        "grid": (cases.grid_graph_2d(64, 64), 4, 1000),
        "hexbox": (cases.hex_pencil(9, 5, 7, 1, seed=3), 6, 200),
    }[case]
    perm, t = recursive_bisection(p.K, p.M, L, leaf)
    perm_s, t_s = cpu.sequential_partition(p.K, p.M, L, leaf)
    assert np.array_equal(perm, perm_s)
    for k in ("parent", "role", "left", "right", "idx_ptr", "idx"):
        assert np.array_equal(t[k], t_s[k]), k
