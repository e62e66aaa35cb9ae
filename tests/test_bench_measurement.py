"""Host logic of bench.py's measurement, without a GPU: the per-category
roofline of the whole solve, and the CPU arm's timed step, which starts with
the reference's partition (AmlsSolver::solve partitions inside the call,
solver.cpp:124-134) and must reproduce the tree it is given."""
import numpy as np
import pytest

import bench
from amls_b200 import cases


class _Ledger:
    """Stands in for the solver handle: algorithmic work per category."""

    def __init__(self, work):
        self.work = work

    def category_work(self):
        return self.work


def test_phase_roofline_sums_roofline_times(monkeypatch):
    monkeypatch.setattr(bench, "fp64_gemm_peak", lambda: 40.0)          # TFLOP/s
    work = {"gemm": (4.0e12, 1.0e9), "tridiag": (1.0e9, 8.0e10), "bisect": (0.0, 0.0)}
    ktimes = {"gemm": (400.0, 20), "tridiag": (100.0, 2), "bisect": (0.0, 0)}   # ms and launches over 2 steps
    out = bench.phase_roofline(ktimes, 2, _Ledger(work), 0.5, {"hbm_gbs": 8000.0})
    g, t = out["per_category"]["gemm"], out["per_category"]["tridiag"]
    assert g["bound"] == "fp64" and g["roof_ms"] == pytest.approx(100.0)      # 4e12 / 40e12 s
    assert g["ms"] == pytest.approx(200.0) and g["frac"] == pytest.approx(0.5)
    assert t["bound"] == "hbm" and t["roof_ms"] == pytest.approx(10.0)       # 8e10 / 8e12 s
    assert t["frac"] == pytest.approx(0.2) and t["launches"] == pytest.approx(1.0)
    assert out["per_category"]["bisect"]["frac"] is None                   # not launched
    assert out["roof_ms"] == pytest.approx(110.0)
    assert out["frac_whole_solve"] == pytest.approx(0.22)


def test_cpu_step_times_the_partition_and_checks_the_tree():
    from oracle import cpu
    p = cases.config_pencil("C1", seed=0)
    _, tree = cpu.sequential_partition(p.K, p.M, 4, 500)
    expect = {k: np.asarray(tree[k], np.int64) for k in ("parent", "left", "right", "idx_ptr", "idx")}
    t, pp, pa, tm = bench.cpu_full_solve(p, 2, 20, 4, expect)
    assert tm["partition"] > 0.0 and t >= tm["partition"]
    assert pp > 0 and pa > 0
    wrong = dict(expect)
    wrong["idx"] = expect["idx"][::-1].copy()                              # a tree the partition does not give
    with pytest.raises(RuntimeError, match="differs from the fixture tree"):
        bench.cpu_full_solve(p, 2, 20, 4, wrong)
