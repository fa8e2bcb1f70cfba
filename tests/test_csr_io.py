"""CPU: the reference's .csr binary format (csr.cuh:119-191, tasks.py:66-72)."""
import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR, load_csr, reference_equal, save_csr


def tasks_py_writer(path, m, n, indptr, indices, data):
    """The byte sequence tasks.py:66-72 writes for a scipy CSR matrix."""
    with open(path, "wb") as fp:
        np.array([len(indices), m, n], dtype=np.int32).tofile(fp)
        np.asarray(indptr, dtype=np.int32).tofile(fp)
        np.asarray(indices, dtype=np.int32).tofile(fp)
        np.asarray(data, dtype=np.float64).tofile(fp)


def test_roundtrip_bytes(tmp_path):
    A = G.uniform_rows(30, 3, seed=1, m=20)
    p = tmp_path / "a.csr"
    save_csr(p, A)
    q = tmp_path / "b.csr"
    tasks_py_writer(q, A.m, A.n, A.rpt, A.col, A.val)
    assert p.read_bytes() == q.read_bytes()
    B = load_csr(p)
    assert (B.m, B.n, B.nnz) == (A.m, A.n, A.nnz)
    assert np.array_equal(B.rpt, A.rpt) and np.array_equal(B.col, A.col)
    assert np.array_equal(B.val, A.val)


def test_float_values_stored_as_double(tmp_path):
    A = G.uniform_rows(10, 2, seed=2).astype(np.float32)
    p = tmp_path / "f.csr"
    save_csr(p, A)
    assert p.stat().st_size == 12 + 4 * (A.m + 1) + 4 * A.nnz + 8 * A.nnz
    B = load_csr(p, np.float32)
    assert B.val.dtype == np.float32 and np.array_equal(B.val, A.val)


def test_size_checks(tmp_path):
    A = G.uniform_rows(10, 2, seed=3)
    p = tmp_path / "a.csr"
    save_csr(p, A)
    data = p.read_bytes()
    (tmp_path / "big.csr").write_bytes(data + b"\0")
    with pytest.raises(ValueError, match="too large"):
        load_csr(tmp_path / "big.csr")
    (tmp_path / "short.csr").write_bytes(data[:-1])
    with pytest.raises(ValueError):
        load_csr(tmp_path / "short.csr")
    (tmp_path / "tiny.csr").write_bytes(b"\0" * 8)
    with pytest.raises(ValueError, match="too small"):
        load_csr(tmp_path / "tiny.csr")


def test_reference_equal_tolerance():
    A = G.uniform_rows(20, 3, seed=4)
    B = HostCSR(A.m, A.n, A.rpt.copy(), A.col.copy(), A.val.copy())
    assert reference_equal(A, B)
    B.val[0] += 1e-9
    assert reference_equal(A, B)
    B.val[0] += 1e-3
    assert not reference_equal(A, B)
    B = HostCSR(A.m, A.n, A.rpt.copy(), A.col.copy(), A.val.copy())
    B.col[0] = (B.col[0] + 1) % A.n
    assert not reference_equal(A, B)
