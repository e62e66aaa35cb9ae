"""CPU tests of the oracle (the CPU restatement of the reference) against the
reference's own known-answer tests and the committed golden fixtures.

Reference KATs restated here:
  tests/unit/test_io.cpp:31-79          closed-form path / grid spectra vs dsygvd
  tests/unit/test_linalg.cpp:16-55      dsygvd / dsygvx index and interval semantics
  tests/unit/test_amls.cpp:41-66        truncation policies
  tests/unit/test_amls.cpp:68-108       condensation structure P3 / P4 / P8
  tests/unit/test_amls.cpp:110-151      keep-all AMLS is exact (1e-10) + back-transform
  tests/regression/test_regression.cpp:29-85  end-to-end 4 % and dense-vs-Lanczos 1e-8
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from amls_b200 import cases
from oracle import amls_ref as R

from .helpers import partition, rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_path_spectrum_closed_form():
    p = cases.path_graph(60)
    w, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    assert rel_err(w, cases.path_graph_spectrum(60)) < 1e-12
    pc = cases.path_graph(40, True)
    w, _ = R.LapackDense.solve_all(pc.K.toarray(), pc.M.toarray())
    assert rel_err(w, cases.path_graph_spectrum(40, True)) < 1e-12


def test_grid_spectra_closed_form():
    p = cases.grid_graph_2d(7, 9)
    w, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    assert rel_err(w, cases.grid_graph_2d_spectrum(7, 9)) < 1e-12
    p = cases.grid_graph_3d(4, 4, 4)
    w, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    assert rel_err(w, cases.grid_graph_3d_spectrum(4, 4, 4)) < 1e-12


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    return A @ A.T + n * np.eye(n), B @ B.T / n + np.eye(n)


def test_dense_eigensolver_semantics():
    K, M = _spd(30, 1)
    w, V = R.LapackDense.solve_all(K, M)
    assert np.allclose(V.T @ M @ V, np.eye(30), atol=1e-10)
    wi, Vi = R.LapackDense.solve_index(K, M, 1, 7)
    assert wi.shape == (7,) and rel_err(wi, w[:7]) < 1e-12
    hi = 0.5 * (w[4] + w[5])
    wv, Vv = R.LapackDense.solve_interval(K, M, -1.0, hi)
    assert wv.shape == (5,) and rel_err(wv, w[:5]) < 1e-12
    # empty interval -> m = 0
    we, Ve = R.LapackDense.solve_interval(K, M, -1.0, -0.5)
    assert we.size == 0 and Ve.shape == (30, 0)


def test_truncation_policies():
    w = np.arange(1.0, 11.0)
    tr = R.FixedCountTruncation(3)
    assert tr.select(w, 10) == 3 and tr.select(w, 2) == 2
    assert tr.index_hint() == (1, 3)
    allk = R.FixedCountTruncation(0)
    assert allk.select(w, 10) == 10 and allk.index_hint() is None
    th = R.ThresholdTruncation(5.5)
    assert th.select(w, 10) == 5
    assert th.interval_hint() == (-1e300, 5.5)
    assert R.ThresholdTruncation(-1.0).select(w, 10) == 0


def test_condensation_structure_p3_p4_p8():
    p = cases.grid_graph_2d(8, 8)
    perm, tree = partition(p, 1, 15)
    Kp, Mp = R.permute_symmetric(p.K, perm), R.permute_symmetric(p.M, perm)
    ge = R.GaussianEliminationRef(Kp, Mp, tree)
    ge.run()
    r = R.SubspaceCondensationRef(ge, R.EigenpairSolverRef()).run(R.FixedCountTruncation(0))
    for i in tree.post_order():                      # P3
        assert len(r.mu[i]) == r.k[i]
        assert np.all(np.diff(r.mu[i]) >= 0)
        assert r.Z[i].shape == (len(tree.indices[i]), r.k[i])
    for (ri, ci, _) in r.mproj_blocks:               # P4
        assert ri in tree.ancestors(ci)
    Mpj = R.assemble_mproj(r)                        # P8
    for i in tree.post_order():
        o, k = r.proj_offset[i], r.k[i]
        assert np.linalg.norm(Mpj[o:o + k, o:o + k] - np.eye(k)) < 1e-10


def test_keep_all_exact_and_backtransform():
    p = cases.grid_graph_2d(10, 10)
    perm, tree = partition(p, 2, 20)
    Kp, Mp = R.permute_symmetric(p.K, perm), R.permute_symmetric(p.M, perm)
    ge = R.GaussianEliminationRef(Kp, Mp, tree)
    ge.run()
    cond = R.SubspaceCondensationRef(ge, R.EigenpairSolverRef())
    r = cond.run(R.FixedCountTruncation(0))
    assert r.p == 100
    w, V = R.LapackDense.solve_all(R.assemble_kproj(r), R.assemble_mproj(r))
    assert rel_err(w[:10], cases.grid_graph_2d_spectrum(10, 10)[:10]) < 1e-10
    z = cond.backtransform(r, V[:, :3])
    Kd, Md = Kp.toarray(), Mp.toarray()
    for j in range(3):
        rz = Kd @ z[:, j] - w[j] * (Md @ z[:, j])
        assert np.linalg.norm(rz) < 1e-10 * np.linalg.norm(Kd @ z[:, j])


def test_regression_path_2000():
    p = cases.path_graph(2000)
    s = R.amls_solve_ref(p.K, p.M, partition(p, 4, 500)[1], R.OptionsRef(nev=50, nLevels=4))
    assert rel_err(s.theta, cases.path_graph_spectrum(2000)[:50]) <= 0.04


def test_regression_path_800_consistent_mass():
    p = cases.path_graph(800, True)
    s = R.amls_solve_ref(p.K, p.M, partition(p, 4, 500)[1], R.OptionsRef(nev=30, nLevels=4))
    assert rel_err(s.theta, cases.path_graph_spectrum(800, True)[:30]) <= 0.04


def test_regression_grid_eta_monotone():
    """test_regression.cpp:54-74 on a smaller grid: eta 2 -> 4 does not worsen."""
    p = cases.grid_graph_2d(24, 24)
    ref = cases.grid_graph_2d_spectrum(24, 24)[:20]
    _, tree = partition(p, 3, 100)
    e = []
    for eta in (2.0, 4.0):
        s = R.amls_solve_ref(p.K, p.M, tree, R.OptionsRef(nev=20, nLevels=3, leafSize=100,
                                                          thresholdFactor=eta, silMode=-1))
        e.append(rel_err(s.theta, ref))
    assert e[1] <= e[0] + 1e-12


def test_dense_vs_lanczos_reference():
    """test_regression.cpp:76-85: dense dsygvd vs shift-invert Lanczos agree to 1e-8."""
    p = cases.path_graph(300)
    w1, _ = R.smallest_eigenpairs(p.K, p.M, 10, dense_max=5000)
    w2, _ = R.smallest_eigenpairs(p.K, p.M, 10, dense_max=0)
    assert rel_err(w2, w1) <= 1e-8


def test_sil_interval_matches_dense_on_sparse_leaf():
    """The SIL kernel (shift_invert_lanczos.hpp) finds the low modes of a
    sparse node pencil; its values agree with dsygvx to Lanczos accuracy.
    Like the reference (its pick loop walks nu ascending, :153-160), the
    interval result comes out in descending order of lambda."""
    p = cases.grid_graph_2d(16, 16)
    K, M = p.K.toarray(), p.M.toarray()
    w, _ = R.LapackDense.solve_interval(K, M, -1e300, 0.3)
    ws, Vs = R.sil_solve_interval(K, M, -1e300, 0.3)
    assert ws.size == w.size
    assert np.all(np.diff(ws) <= 0)
    assert rel_err(np.sort(ws), w) < 1e-8


def test_golden_fixtures():
    """The oracle reproduces the committed golden vectors
    (tests/golden/make_golden.py)."""
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        meta = json.load(f)
    for name, m in meta.items():
        data = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        p = _golden_pencil(m["pencil"])
        perm, tree = partition(p, m["nLevels"], m["leafSize"])
        assert np.array_equal(perm, data["perm"]), name
        s = R.amls_solve_ref(p.K, p.M, tree, R.OptionsRef(silMode=-1, nev=m["nev"],
                                                           nLevels=m["nLevels"],
                                                           leafSize=m["leafSize"]))
        assert s.p == int(data["p"]), name
        assert rel_err(s.theta, data["theta"]) < 1e-12, name


def _golden_pencil(spec):
    kind = spec[0]
    if kind == "hex":
        return cases.hex_pencil(*spec[1:4], spec[4], seed=spec[5])
    if kind == "grid":
        return cases.grid_graph_2d(spec[1], spec[2])
    if kind == "path":
        return cases.path_graph(spec[1], bool(spec[2]))
    raise ValueError(kind)


def test_permute_symmetric_convention():
    p = cases.grid_graph_2d(6, 5)
    perm, tree = partition(p, 2, 8)
    B = R.permute_symmetric(p.K, perm)
    A = p.K.toarray()
    assert np.array_equal(B.toarray(), A[np.ix_(perm, perm)])
    assert sp.issparse(B)


def test_reference_start_vector_generator():
    """The SIL start vector: std::srand / std::rand of the Microsoft C
    runtime (first values after srand(1) are the documented 41, 18467, 6334,
    26500, 19169) mapped to [-1, 1] as Eigen 3.4's Random does."""
    assert R.msvcrt_rand(1, 5).tolist() == [41, 18467, 6334, 26500, 19169]
    v = R.reference_start_vector(1000)
    assert v.min() >= -1.0 and v.max() <= 1.0
    r = R.msvcrt_rand(12345, 3)
    assert np.allclose(v[:3], -1.0 + 2.0 * r / 32767.0)
