"""Matrix Market IO through the C ABI (host only): the reference's
round trip to 1e-14 (tests/unit/test_io.cpp:19-29), symmetric expansion,
pattern and integer fields, comments, duplicates summed, bad files refused."""
import numpy as np
import pytest
import scipy.sparse as sp

from amls_b200 import cases, read_matrix_market, write_matrix_market


def test_round_trip_grid(tmp_path):
    p = cases.grid_graph_2d(12, 9)
    f = tmp_path / "K.mtx"
    write_matrix_market(f, p.K)
    A = read_matrix_market(f)
    assert A.shape == p.K.shape
    assert abs(A - p.K).max() <= 1e-14 * abs(p.K).max()
    assert open(f).readline().startswith("%%MatrixMarket matrix coordinate real symmetric")


def test_round_trip_hex(tmp_path):
    p = cases.hex_pencil(3, 3, 2, 2, seed=1)
    f = tmp_path / "M.mtx"
    write_matrix_market(f, p.M)
    A = read_matrix_market(f)
    assert abs(A - p.M).max() <= 1e-14 * abs(p.M).max()


def test_fields_symmetry_duplicates(tmp_path):
    f = tmp_path / "a.mtx"
    f.write_text("%%MatrixMarket matrix coordinate integer general\n% comment\n\n3 3 4\n"
                 "1 1 2\n2 1 -1\n2 1 -1\n3 3 5\n")
    A = read_matrix_market(f).toarray()
    assert np.array_equal(A, np.array([[2, 0, 0], [-2, 0, 0], [0, 0, 5]], float))
    g = tmp_path / "b.mtx"
    g.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n1 1\n3 1\n2 2\n")
    B = read_matrix_market(g).toarray()
    assert np.array_equal(B, np.array([[1, 0, 1], [0, 1, 0], [1, 0, 0]], float))


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n",
    "not a banner\n",
    "%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1\n",
])
def test_bad_files_refused(tmp_path, text):
    f = tmp_path / "bad.mtx"
    f.write_text(text)
    with pytest.raises(ValueError):
        read_matrix_market(f)
