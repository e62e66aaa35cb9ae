"""GPU parity tests through the C ABI: the CUDA path against the oracle
(the CPU restatement of the reference) and against known answers.

Tolerances: eigenvalues of the plain FP64 path within 1e-10 relative of the
oracle's theta on the same input (same partition, same truncation); the
keep-all case within 1e-10 of the closed-form spectrum
(tests/unit/test_amls.cpp:110-151 of the reference); dense eigensolver
within 1e-12 relative of LAPACK dsygvx (tests/unit/test_linalg.cpp:16-55).
"""
import numpy as np
import pytest
import scipy.linalg as sla

from amls_b200 import AmlsOptions, NotSPDError, cases, sygvx_batched
from oracle import amls_ref as R

from .helpers import oracle_solve, rel_err, residuals

pytestmark = pytest.mark.gpu


def _rand_pencil(n, rng):
    A = rng.standard_normal((n, n))
    K = A @ A.T + n * np.eye(n)
    B = rng.standard_normal((n, n))
    M = B @ B.T / n + np.eye(n)
    return K, M


@pytest.mark.parametrize("n", [1, 2, 7, 40, 200, 383, 390, 700])
def test_sygvx_index_matches_lapack(solver, n):
    rng = np.random.default_rng(n)
    K, M = _rand_pencil(n, rng)
    k = min(n, 12)
    (w, V), = sygvx_batched(solver, [K], [M], mode="index", il=1, iu=k)
    wr, Vr = R.LapackDense.solve_index(K, M, 1, k)
    assert w.shape == wr.shape
    assert rel_err(w, wr) < 1e-12
    # M-orthonormal, residual small
    assert np.allclose(V.T @ M @ V, np.eye(k), atol=1e-10)
    res = np.linalg.norm(K @ V - M @ V * w[None, :], axis=0) / np.linalg.norm(K, 1)
    assert res.max() < 1e-12


def test_sygvx_many_large_in_chunks(solver):
    """More matrices above the one-CTA size than SMs: the cooperative
    tridiagonalisation runs in several launches; plus one matrix of order
    1,500 sharing a launch with smaller ones."""
    rng = np.random.default_rng(11)
    sizes = [390 + (i % 7) for i in range(150)] + [1500]
    Ks, Ms = zip(*[_rand_pencil(n, rng) for n in sizes])
    out = sygvx_batched(solver, list(Ks), list(Ms), mode="index", il=1, iu=3)
    for b in list(range(0, 150, 37)) + [149, 150]:
        wr, _ = R.LapackDense.solve_index(Ks[b], Ms[b], 1, 3)
        assert rel_err(out[b][0], wr) < 1e-12


def test_sygvx_interval_batched_uneven(solver):
    rng = np.random.default_rng(5)
    sizes = [3, 17, 64, 150, 420]
    Ks, Ms = zip(*[_rand_pencil(n, rng) for n in sizes])
    hi = 1.5 * np.median([sla.eigh(K, M, eigvals_only=True)[2] for K, M in zip(Ks, Ms)])
    out = sygvx_batched(solver, list(Ks), list(Ms), mode="interval", lo=-1e300, hi=hi)
    for (w, V), K, M in zip(out, Ks, Ms):
        wr, _ = R.LapackDense.solve_interval(K, M, -1e300, hi)
        assert w.shape == wr.shape            # same count in (lo, hi]
        if w.size:
            assert rel_err(w, wr) < 1e-12


def test_keep_all_is_exact_grid(solver):
    """Keep-all AMLS reproduces the closed-form 10x10 grid spectrum
    (reference tests/unit/test_amls.cpp:110-151)."""
    p = cases.grid_graph_2d(10, 10)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=10, nLevels=2, leafSize=20, fixedKeep=10 ** 6))
    ref = cases.grid_graph_2d_spectrum(10, 10)[:10]
    assert sol.p == 100
    assert rel_err(sol.theta, ref) < 1e-10
    assert residuals(p.K, p.M, sol.theta, sol.Z)[:3].max() < 1e-10


def test_keep_all_is_exact_hex(solver):
    p = cases.hex_pencil(4, 4, 4, 1, seed=3)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=15, nLevels=3, leafSize=60, fixedKeep=10 ** 6))
    wr, _ = R.smallest_eigenpairs(p.K, p.M, 15)
    assert rel_err(sol.theta, wr) < 1e-10


@pytest.mark.parametrize("case", ["hex8_5", "grid_40", "path_600"])
def test_two_pass_matches_oracle(solver, case):
    if case == "hex8_5":
        p = cases.hex_pencil(5, 5, 5, 1, seed=1)
        o = dict(nev=20, nLevels=3, leafSize=100)
    elif case == "grid_40":
        p = cases.grid_graph_2d(40, 40)
        o = dict(nev=30, nLevels=4, leafSize=150)
    else:
        p = cases.path_graph(600, True)
        o = dict(nev=25, nLevels=4, leafSize=60)
    ref = oracle_solve(p, R.OptionsRef(silMode=-1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(**o))
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10
    # vectors: same Ritz pairs up to sign -> compare residuals and M-norms
    r = residuals(p.K, p.M, sol.theta, sol.Z)
    rr = residuals(p.K, p.M, ref.theta, ref.Z)
    assert np.all(r < 10 * rr + 1e-12)
    mn = np.einsum("ij,ij->j", sol.Z, p.M @ sol.Z)
    assert np.allclose(mn, 1.0, atol=1e-12)


def test_c1_matches_oracle(solver):
    """Config C1: 8-node hex 12^3 (6,084 DOF), L = 4, nev = 20."""
    p = cases.config_pencil("C1")
    o = dict(nev=20, nLevels=4, leafSize=500)
    ref = oracle_solve(p, R.OptionsRef(silMode=-1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(**o))
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10


def test_fixed_keep_matches_oracle(solver):
    p = cases.hex_pencil(6, 5, 4, 1, seed=7)
    o = dict(nev=12, nLevels=3, leafSize=80, fixedKeep=6)
    ref = oracle_solve(p, R.OptionsRef(silMode=-1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(**o))
    assert sol.p == ref.p
    assert rel_err(sol.theta, ref.theta) < 1e-10


def test_shift_matches_oracle(solver):
    p = cases.hex_pencil(4, 4, 5, 1, seed=2)
    o = dict(nev=10, nLevels=3, leafSize=60, shift=0.5)
    ref = oracle_solve(p, R.OptionsRef(silMode=-1, **o))
    sol = solver.solve(p.K, p.M, AmlsOptions(**o))
    assert rel_err(sol.theta, ref.theta) < 1e-10


def test_not_spd_raises(solver):
    """A non-SPD K is reported as NotSPDError (reference P10 check), and the
    handle stays usable afterwards."""
    p = cases.hex_pencil(3, 3, 3, 1, seed=0)
    K = p.K.copy()
    K.data = -K.data
    with pytest.raises(NotSPDError):
        solver.solve(K, p.M, AmlsOptions(nev=5, nLevels=2, leafSize=30))
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=5, nLevels=2, leafSize=30, fixedKeep=10 ** 6))
    wr, _ = R.smallest_eigenpairs(p.K, p.M, 5)
    assert rel_err(sol.theta, wr) < 1e-10


def test_invalid_arguments(solver):
    p = cases.path_graph(50)
    with pytest.raises(ValueError):
        solver.solve(p.K, p.M, AmlsOptions(nev=0))
    with pytest.raises(ValueError):
        solver.solve(p.K, p.M, AmlsOptions(nev=5, twoPass=False))


def test_c5_matches_oracle_golden(solver):
    """Full-size workload (27-node hex 14^3, 70,644 DOF, nev 500, L 8): the
    GPU theta equal the oracle's golden theta (tests/golden/make_c5_golden.py)
    within 1e-10, with the same reduced sizes."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c5_oracle.npz"))
    p = cases.config_pencil("C5", seed=0)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=500, nLevels=8, leafSize=500,
                                             recoverVectors=False))
    assert np.array_equal(solver.permutation(), g["perm"])     # same partition and tree order
    assert sol.p == int(g["p"])
    assert sol.info["p_passA"] == int(g["p_passA"])
    assert rel_err(sol.theta, g["theta"]) < 1e-10


@pytest.mark.parametrize("case,refine", [("hex8_8", 1), ("hex8_8", 3), ("hex27_4", 3)])
def test_refinement_reaches_exact_eigenvalues(solver, case, refine):
    """FP64 refinement (subspace iteration with the elimination's exact K
    factorisation + Rayleigh-Ritz) brings the AMLS Ritz values to the exact
    eigenvalues: relative error <= 1e-8 against dense LAPACK dsygvd."""
    if case == "hex8_8":
        p = cases.hex_pencil(8, 8, 8, 1, seed=5)
        o = dict(nev=40, nLevels=4, leafSize=200)
    else:
        p = cases.hex_pencil(4, 4, 4, 2, seed=6)
        o = dict(nev=30, nLevels=4, leafSize=200)
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    plain = solver.solve(p.K, p.M, AmlsOptions(**o))
    sol = solver.solve(p.K, p.M, AmlsOptions(refine=refine, **o))
    assert rel_err(plain.theta, wr[:o["nev"]]) > 1e-6          # AMLS alone is approximate
    assert rel_err(sol.theta, wr[:o["nev"]]) < 1e-8
    assert sol.info["refine_iters"] >= 1
    assert residuals(p.K, p.M, sol.theta, sol.Z).max() < 1e-6
    mn = np.einsum("ij,ij->j", sol.Z, p.M @ sol.Z)
    assert np.allclose(mn, 1.0, atol=1e-12)


def test_c5_refined_matches_exact(solver):
    """Full-size workload with FP64 refinement: all 500 eigenvalues within
    1e-8 relative of the exact ones (shift-invert Lanczos golden,
    tests/golden/make_c5_golden.py)."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c5_exact.npz"))["theta"]
    p = cases.config_pencil("C5", seed=0)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=500, nLevels=8, leafSize=500, refine=3,
                                             recoverVectors=False))
    assert rel_err(sol.theta, g[:500]) < 1e-8


def test_c5_refined_high_filter_degree(solver):
    """A degree-4 Chebyshev filter (refine = 5) makes the filtered block of
    the full-size workload lose rank; the refinement lowers the degree and
    still reaches the exact eigenvalues."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c5_exact.npz"))["theta"]
    p = cases.config_pencil("C5", seed=0)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=500, nLevels=8, leafSize=500, refine=5,
                                             recoverVectors=False))
    assert rel_err(sol.theta, g[:500]) < 1e-8


@pytest.mark.parametrize("case", ["hex8_8", "hex27_4"])
def test_mixed_precision_amls_close_to_fp64(solver, case):
    """Mixed precision (M-side AMLS products on the BF16 tensor cores with
    split operands, relative error ~2^-16 per product): the AMLS Ritz values
    move by far less than the AMLS truncation error itself."""
    if case == "hex8_8":
        p = cases.hex_pencil(8, 8, 8, 1, seed=5)
        o = dict(nev=40, nLevels=4, leafSize=200)
    else:
        p = cases.hex_pencil(4, 4, 4, 2, seed=6)
        o = dict(nev=30, nLevels=4, leafSize=200)
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    f64 = solver.solve(p.K, p.M, AmlsOptions(**o))
    mix = solver.solve(p.K, p.M, AmlsOptions(precision="mixed", **o))
    assert f64.p == mix.p
    trunc = rel_err(f64.theta, wr[:o["nev"]])
    assert rel_err(mix.theta, f64.theta) < 1e-3 * max(trunc, 1e-6) + 1e-4


@pytest.mark.parametrize("case", ["hex8_8", "hex27_4"])
def test_mixed_precision_refined_reaches_exact(solver, case):
    """Mixed precision followed by the FP64 refinement: eigenvalues within
    1e-8 relative of dense LAPACK dsygvd, M-normalised vectors."""
    if case == "hex8_8":
        p = cases.hex_pencil(8, 8, 8, 1, seed=5)
        o = dict(nev=40, nLevels=4, leafSize=200)
    else:
        p = cases.hex_pencil(4, 4, 4, 2, seed=6)
        o = dict(nev=30, nLevels=4, leafSize=200)
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    sol = solver.solve(p.K, p.M, AmlsOptions(precision="mixed", refine=3, **o))
    assert rel_err(sol.theta, wr[:o["nev"]]) < 1e-8
    assert residuals(p.K, p.M, sol.theta, sol.Z).max() < 1e-6
    mn = np.einsum("ij,ij->j", sol.Z, p.M @ sol.Z)
    assert np.allclose(mn, 1.0, atol=1e-12)


def test_c5_mixed_refined_matches_exact(solver):
    """Full-size workload, mixed precision + FP64 refinement: all 500
    eigenvalues within 1e-8 relative of the exact golden."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c5_exact.npz"))["theta"]
    p = cases.config_pencil("C5", seed=0)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=500, nLevels=8, leafSize=500, refine=3,
                                             precision="mixed", recoverVectors=False))
    assert rel_err(sol.theta, g[:500]) < 1e-8


def test_invalid_precision(solver):
    p = cases.hex_pencil(3, 3, 3, 1, seed=1)
    with pytest.raises(ValueError):
        solver.solve(p.K, p.M, AmlsOptions(nev=5, nLevels=2, precision="fp16"))


def test_elimination_graph_replay_matches_eager(solver):
    """The numeric solve replays the elimination and the refinement's K^-1 M
    applications as captured CUDA graphs (with per-launch instrumentation
    off); it gives the eager launches' eigenvalues (up to the order of the
    extend-add and split-K atomics), also on repeat."""
    p = cases.hex_pencil(8, 8, 8, 1, seed=5)
    o = AmlsOptions(nev=40, nLevels=4, leafSize=200, refine=3)
    solver.analyze(p.K, p.M, o)
    kv = np.ascontiguousarray(p.K.data)
    mv = np.ascontiguousarray(p.M.data)
    th = [np.zeros(40) for _ in range(3)]
    solver.set_profiling(True)           # eager launches, an event pair around each
    solver.solve_values(kv.ctypes.data, mv.ctypes.data, False, th[0].ctypes.data, None, False)
    solver.set_profiling(False)          # captured at the second solve, then replayed
    for t in th[1:]:
        solver.solve_values(kv.ctypes.data, mv.ctypes.data, False, t.ctypes.data, None, False)
    assert rel_err(th[1], th[0]) < 1e-12
    assert rel_err(th[2], th[0]) < 1e-12
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    assert rel_err(th[2], wr[:40]) < 1e-8


def _golden(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name))


def test_c2_fp64_matches_oracle_golden(solver):
    """Precision workload (27-node hex 7^3, 9,450 DOF, nev 100, reference
    defaults nLevels 6, leafSize 500, eta 2): the plain FP64 GPU theta equal
    the oracle's (tests/golden/make_c2c4_golden.py) within 1e-10, same
    permutation and reduced sizes."""
    g = _golden("c2_oracle.npz")
    p = cases.config_pencil("C2", seed=0)
    sol = solver.solve(p.K, p.M, AmlsOptions(nev=100, nLevels=6, leafSize=500, recoverVectors=False))
    assert np.array_equal(solver.permutation(), g["perm"])
    assert sol.p == int(g["p"])
    assert sol.info["p_passA"] == int(g["p_passA"])
    assert rel_err(sol.theta, g["theta"]) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c2_per_eigenvalue_error_against_exact(solver, precision):
    """Precision workload, mixed (BF16-split tensor-core M-side products) and
    FP64: per-eigenvalue relative error against the exact eigenvalues
    (shift-invert Lanczos, the reference's ReferenceSolver path above 5,000
    DOF).  Unrefined: the AMLS truncation error (a few per cent) dominates
    and the two precisions agree to 1e-4 of it; refined: every eigenvalue
    within 1e-8, residuals small, vectors M-normalised."""
    ex = _golden("c2_exact.npz")["theta"][:100]
    p = cases.config_pencil("C2", seed=0)
    o = dict(nev=100, nLevels=6, leafSize=500)
    plain64 = solver.solve(p.K, p.M, AmlsOptions(recoverVectors=False, **o))
    plain = solver.solve(p.K, p.M, AmlsOptions(precision=precision, recoverVectors=False, **o))
    err_plain = np.abs(plain.theta - ex) / ex
    trunc = np.abs(plain64.theta - ex) / ex
    assert np.all(err_plain < 0.15)                          # AMLS alone: approximate
    assert rel_err(plain.theta, plain64.theta) < 1e-4 * trunc.max() + 1e-12
    ref = solver.solve(p.K, p.M, AmlsOptions(precision=precision, refine=3, refineTol=1e-10, **o))
    err = np.abs(ref.theta - ex) / ex
    assert err.max() < 1e-8, (precision, err.max(), int(np.argmax(err)))
    assert residuals(p.K, p.M, ref.theta, ref.Z).max() < 1e-6
    mn = np.einsum("ij,ij->j", ref.Z, p.M @ ref.Z)
    assert np.allclose(mn, 1.0, atol=1e-12)


def test_device_graph_partition_equals_host_partition(solver):
    """The engine builds the graph of |K| + |M| on the GPU for METIS; the
    permutation equals the host partitioner's on the same pencil."""
    from amls_b200.solver import recursive_bisection
    for p, L, leaf in ((cases.config_pencil("C1"), 4, 500), (cases.grid_graph_2d(40, 30), 4, 150),
                       (cases.hex_pencil(5, 6, 4, 2, seed=2), 5, 300)):
        perm, _ = recursive_bisection(p.K, p.M, L, leaf)
        solver.analyze(p.K, p.M, AmlsOptions(nev=5, nLevels=L, leafSize=leaf))
        assert np.array_equal(solver.permutation(), perm)
