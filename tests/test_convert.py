"""Real-matrix ingest (no GPU): Matrix Market and SuiteSparse .mat files to
the .csr format, checked against scipy's readers and the .csr round trip."""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from gpuspgemm_b200.convert import convert, main, read_mtx
from gpuspgemm_b200.csr import load_csr


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return p


def _same_as_scipy(a, ref):
    ref = sp.csr_matrix(ref)
    ref.sum_duplicates()
    ref.sort_indices()
    assert (a.m, a.n) == ref.shape
    assert np.array_equal(a.rpt, ref.indptr)
    assert np.array_equal(a.col, ref.indices)
    assert np.allclose(a.val, ref.data, rtol=0, atol=0)


@pytest.mark.parametrize("field,symmetry", [("real", "general"), ("integer", "general"),
                                            ("pattern", "general"), ("real", "symmetric"),
                                            ("real", "skew-symmetric"), ("pattern", "symmetric")])
def test_mtx_matches_scipy(tmp_path, field, symmetry):
    rng = np.random.default_rng(7)
    m = n = 40
    rows = rng.integers(0, m, 150)
    cols = rng.integers(0, n, 150)
    if symmetry != "general":  # lower triangle only; strict for skew
        lo = np.minimum(rows, cols)
        hi = np.maximum(rows, cols)
        rows, cols = hi, lo
        if symmetry == "skew-symmetric":
            keep = rows != cols
            rows, cols = rows[keep], cols[keep]
    vals = rng.integers(-5, 6, rows.size) if field == "integer" else rng.uniform(-1, 1, rows.size)
    lines = [f"%%MatrixMarket matrix coordinate {field} {symmetry}", "% a comment",
             f"{m} {n} {rows.size}"]
    for r, c, v in zip(rows, cols, vals):
        lines.append(f"{r + 1} {c + 1}" if field == "pattern" else f"{r + 1} {c + 1} {float(v)!r}")
    p = _write(tmp_path, "a.mtx", "\n".join(lines) + "\n")
    a = read_mtx(p)
    _same_as_scipy(a, scipy.io.mmread(p))


def test_mtx_duplicates_summed_and_zeros_kept(tmp_path):
    p = _write(tmp_path, "d.mtx", "%%MatrixMarket matrix coordinate real general\n"
               "3 4 5\n1 2 1.5\n1 2 2.5\n3 4 0.0\n2 1 -1\n% trailing comment\n1 1 7\n")
    a = read_mtx(p)
    assert a.rpt.tolist() == [0, 2, 3, 4]
    assert a.col.tolist() == [0, 1, 0, 3]
    assert a.val.tolist() == [7.0, 4.0, -1.0, 0.0]


def test_mtx_rejects_unsupported(tmp_path):
    bad = [("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "coordinate"),
           ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "complex"),
           ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n", "expected"),
           ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", "outside")]
    for text, msg in bad:
        with pytest.raises(ValueError, match=msg):
            read_mtx(_write(tmp_path, "x.mtx", text))


def test_mat_and_csr_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    A = sp.random(50, 30, density=0.1, random_state=4, format="csc")
    problem = {"A": A, "name": "test/random"}
    src = tmp_path / "p.mat"
    scipy.io.savemat(src, {"Problem": problem})
    out = tmp_path / "p.csr"
    assert main([str(src), str(out)]) == 0
    a = load_csr(out)
    _same_as_scipy(a, A.tocsr())
    # the file layout: int32 nnz, m, n; rpt; col; float64 values
    raw = out.read_bytes()
    assert len(raw) == 12 + 4 * (a.m + 1) + 4 * a.nnz + 8 * a.nnz
    # .mtx -> .csr through the same entry point
    m = tmp_path / "p.mtx"
    scipy.io.mmwrite(m, A)
    b = convert(m, tmp_path / "q.csr")
    assert np.array_equal(b.col, a.col) and np.allclose(b.val, a.val)
    del rng
