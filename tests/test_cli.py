"""The command-line programs amls_solve / amls_verify (the reference's
src/apps/amls_solve.cpp and amls_verify.cpp flags and outputs): usage
errors on the CPU; solves and the closed-form verification sweep on the
GPU."""
import os
import subprocess

import numpy as np
import pytest

from amls_b200 import cases, write_matrix_market

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOLVE = os.path.join(HERE, "amls_b200", "amls_solve")
VERIFY = os.path.join(HERE, "amls_b200", "amls_verify")


def _run(args, **kw):
    return subprocess.run(args, capture_output=True, text=True, timeout=600, **kw)


def test_usage_errors():
    assert _run([SOLVE]).returncode == 2
    assert _run([SOLVE, "--case", "path"]).returncode == 2
    assert _run([SOLVE, "--case", "path:10", "--nev", "x"]).returncode == 2
    assert _run([SOLVE, "--case", "path:10", "--precision", "fp16"]).returncode == 2
    assert _run([VERIFY, "--bogus"]).returncode == 2


@pytest.mark.gpu
def test_solve_closed_form_case(tmp_path):
    out = tmp_path / "theta.txt"
    r = _run([SOLVE, "--case", "grid:30,30", "--nev", "12", "--nlevels", "3", "--leaf-size", "120",
              "--fixed-keep", "1000000", "--out", str(out)])
    assert r.returncode == 0, r.stderr
    assert "relerr=" in r.stdout and "# residuals:" in r.stdout
    th = np.loadtxt(out)[:, 1]
    ref = cases.grid_graph_2d_spectrum(30, 30)[:12]
    assert np.max(np.abs(th - ref) / ref) < 1e-10                # keep-all AMLS is exact


@pytest.mark.gpu
def test_solve_matrix_market_pencil(tmp_path):
    p = cases.hex_pencil(4, 4, 4, 1, seed=2)
    write_matrix_market(tmp_path / "K.mtx", p.K)
    write_matrix_market(tmp_path / "M.mtx", p.M)
    out = tmp_path / "t.txt"
    r = _run([SOLVE, "--K", str(tmp_path / "K.mtx"), "--M", str(tmp_path / "M.mtx"), "--nev", "8",
              "--nlevels", "3", "--leaf-size", "60", "--refine", "3", "--out", str(out)])
    assert r.returncode == 0, r.stderr
    from oracle import amls_ref as R
    wr, _ = R.LapackDense.solve_all(p.K.toarray(), p.M.toarray())
    th = np.loadtxt(out)[:, 1]
    assert np.max(np.abs(th - wr[:8]) / wr[:8]) < 1e-8


@pytest.mark.gpu
def test_verify_closed_quick(tmp_path):
    r = _run([VERIFY, "--suite", "closed", "--quick", "--outdir", str(tmp_path)])
    assert r.returncode == 0, r.stdout + r.stderr
    csv = (tmp_path / "verify_results.csv").read_text().splitlines()
    assert csv[0].startswith("case,eta,nLevels,p,maxRelErr")
    assert len(csv) == 1 + 4 and all(line.endswith(",1") for line in csv[1:])
    assert "passed 4/4" in (tmp_path / "verify_report.md").read_text()
