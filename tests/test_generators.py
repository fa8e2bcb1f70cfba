"""CPU: seeded synthetic inputs have the stated shapes and are deterministic."""
import numpy as np

from gpuspgemm_b200 import generators as G


def test_uniform_rows_exact_degree():
    A = G.uniform_rows(4096, 8)
    A.validate()
    assert A.m == A.n == 4096 and A.nnz == 32768
    assert np.all(np.diff(A.rpt) == 8)
    assert A.val.min() >= -1 and A.val.max() <= 1
    B = G.uniform_rows(4096, 8)
    assert np.array_equal(A.col, B.col) and np.array_equal(A.val, B.val)


def test_power_law_shape():
    A = G.power_law(20000, 2.0, 500, seed=7)
    A.validate()
    deg = np.diff(A.rpt)
    assert deg.min() >= 1 and deg.max() <= 500
    # Zipf(2) mean on [1, 500] is about 4.2; duplicates drop a few entries
    assert 3.0 < deg.mean() < 5.0
    assert A.val.min() > 0 and A.val.max() <= 1
    B = G.power_law(20000, 2.0, 500, seed=7)
    assert np.array_equal(A.col, B.col)


def test_stencil_and_prolongator():
    A = G.stencil27(6)
    A.validate()
    assert A.nnz == (3 * 6 - 2) ** 3
    assert np.all(A.val[A.col == np.repeat(np.arange(A.m), np.diff(A.rpt))] == 26.0)
    P = G.aggregation_prolongator(6)
    P.validate()
    assert P.n == 8 and np.all(np.diff(P.rpt) <= 8) and np.all(np.diff(P.rpt) >= 1)
    R = G.transpose(P)
    R.validate()
    assert (R.m, R.n, R.nnz) == (P.n, P.m, P.nnz)


def test_batch_pairs():
    pairs = list(G.batch_pairs(5, seed=3))
    for A, B in pairs:
        A.validate()
        B.validate()
        assert A.m == A.n == B.m == B.n
        assert 64 <= A.m <= 16384
