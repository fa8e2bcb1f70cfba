"""GPU: CSR transpose and the Galerkin triple product R * (A * P).

Transpose moves values without arithmetic, so it is compared bit for bit
(row pointers, sorted columns and values) with the oracle's stable counting
sort.  R * (A * P) is two chained products: structure bit-exact, values within
1e-12 of the oracle's chain relative to the magnitude bound
(|R| (|A| |P|))_ij -- the stencil's rows sum to zero, so entries cancel and a
plain relative error is not meaningful there.
"""
import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def _heavy_column(m=60_000, n=60, seed=1):
    """A column with > 16384 entries (the global sort bin) beside short ones."""
    rows = np.arange(m)
    col = np.where(rows % 3 == 0, 7, rows % 50).astype(np.int32)
    return HostCSR(m, n, np.arange(m + 1, dtype=np.int32), col,
                   np.random.default_rng(seed).uniform(-1, 1, m))


CASES = {
    "prolongator12": lambda: G.aggregation_prolongator(12),
    "powerlaw30000": lambda: G.power_law(30000, 2.0, 3000, seed=21),
    "rect500x40": lambda: G.uniform_rows(40, 3, seed=3, m=500),
    "wide300x70000": lambda: G.uniform_rows(70_000, 40, seed=4, m=300),
    "heavy_column": _heavy_column,
}


def _gpu_transpose(A, handle, dtype=np.float64):
    from gpuspgemm_b200.api import DeviceCSR, transpose
    return transpose(DeviceCSR.from_host(A.astype(dtype)), handle).to_host()


def _assert_same(T, R):
    assert (T.m, T.n) == (R.m, R.n)
    assert np.array_equal(T.rpt, R.rpt)
    assert np.array_equal(T.col, R.col)
    assert np.array_equal(T.val, R.val)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_transpose_bit_exact(handle, oracle_mod, name, dtype):
    A = CASES[name]().astype(dtype)
    _assert_same(_gpu_transpose(A, handle, dtype), oracle_mod.transpose(A))


@pytest.mark.parametrize("b", range(4))
def test_transpose_forced_bins(handle, oracle_mod, b):
    """Every row of A^T routed to at least sort bin b: each kernel variant
    sorts rows of every length up to its capacity."""
    from gpuspgemm_b200 import _native as N
    assert len(handle.ladder(3, 8)) == 4
    A = G.power_law(3000, 2.0, 300, seed=41)
    handle.set_option(N.OPT_MIN_TRANSPOSE_BIN, b)
    try:
        T = _gpu_transpose(A, handle)
    finally:
        handle.set_option(N.OPT_MIN_TRANSPOSE_BIN, -1)
    _assert_same(T, oracle_mod.transpose(A))


def test_transpose_edge_cases(handle, oracle_mod):
    empty = HostCSR(5, 7, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    T = _gpu_transpose(empty, handle)
    assert (T.m, T.n, T.nnz) == (7, 5, 0) and np.all(T.rpt == 0)
    no_rows = HostCSR(0, 4, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    T = _gpu_transpose(no_rows, handle)
    assert (T.m, T.n, T.nnz) == (4, 0, 0)
    # empty rows and columns in between
    A = HostCSR(4, 6, np.array([0, 2, 2, 5, 5], np.int32),
                np.array([1, 4, 0, 1, 5], np.int32), np.array([1.0, 2.0, 3.0, 4.0, 5.0]))
    _assert_same(_gpu_transpose(A, handle), oracle_mod.transpose(A))
    # transposing twice gives A back
    B = G.power_law(5000, 2.0, 400, seed=8)
    from gpuspgemm_b200.api import DeviceCSR, transpose
    BB = transpose(transpose(DeviceCSR.from_host(B), handle), handle).to_host()
    _assert_same(BB, B)


def test_transpose_rejects_out_of_range_column(handle):
    from gpuspgemm_b200 import SpgemmError
    from gpuspgemm_b200 import _native as N
    A = HostCSR(2, 3, np.array([0, 1, 2], np.int32), np.array([0, 5], np.int32),
                np.array([1.0, 2.0]))
    with pytest.raises(SpgemmError, match="INVALID_ARG"):  # skipped column: count falls short
        _gpu_transpose(A, handle)
    handle.set_option(N.OPT_CHECKED, 1)
    try:
        with pytest.raises(SpgemmError, match="INVALID_ARG"):
            _gpu_transpose(A, handle)
    finally:
        handle.set_option(N.OPT_CHECKED, 0)


def _chain_reference(oracle_mod, R, A, P):
    AP = oracle_mod.spgemm(A, P)
    C = oracle_mod.spgemm(R, AP)
    absd = lambda M: HostCSR(M.m, M.n, M.rpt, M.col, np.abs(M.val.astype(np.float64)))  # noqa: E731
    bound = oracle_mod.spgemm(absd(R), oracle_mod.spgemm(absd(A), absd(P)))
    return C, bound


@pytest.mark.parametrize("given_r", [False, True])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_galerkin_rap(handle, oracle_mod, given_r, dtype):
    from gpuspgemm_b200.api import DeviceCSR, rap
    A = G.stencil27(15).astype(dtype)
    P = G.aggregation_prolongator(15, seed=5).astype(dtype)
    R = oracle_mod.transpose(P)
    dA, dP = DeviceCSR.from_host(A), DeviceCSR.from_host(P)
    dR = DeviceCSR.from_host(R) if given_r else None
    C = rap(dA, dP, dR, handle).to_host()
    ref, bound = _chain_reference(oracle_mod, R.astype(np.float64), A.astype(np.float64),
                                  P.astype(np.float64))
    assert (C.m, C.n) == (P.n, P.n)
    assert np.array_equal(C.rpt, ref.rpt) and np.array_equal(C.col, ref.col)
    err = np.abs(C.val.astype(np.float64) - ref.val) / bound.val
    tol = 1e-12 if dtype == np.float64 else 1e-5
    assert float(err.max()) <= tol, float(err.max())
    info = handle.info()
    assert info["nip"] == oracle_mod.nip(A, P) + oracle_mod.nip(R, oracle_mod.spgemm(A, P))


def test_galerkin_rap_stencil100(handle, oracle_mod):
    """The Galerkin workload at its stated size: 27-point stencil on 100^3
    (1e6 rows, 26.5 M nnz), aggregation prolongator P (1e6 x 35,937), R = P^T
    on the device; R * (A * P) against the oracle chain."""
    from gpuspgemm_b200.api import DeviceCSR, rap
    A = G.stencil27(100)
    P = G.aggregation_prolongator(100, seed=5)
    assert A.nnz == 298 ** 3
    dA, dP = DeviceCSR.from_host(A), DeviceCSR.from_host(P)
    C = rap(dA, dP, None, handle).to_host()
    del dA, dP
    R = oracle_mod.transpose(P)
    ref, bound = _chain_reference(oracle_mod, R, A, P)
    assert (C.m, C.n) == (P.n, P.n)
    assert np.array_equal(C.rpt, ref.rpt) and np.array_equal(C.col, ref.col)
    err = np.abs(C.val - ref.val) / bound.val
    assert float(err.max()) <= 1e-12, float(err.max())


def test_rap_dimension_checks(handle):
    from gpuspgemm_b200 import SpgemmError
    from gpuspgemm_b200.api import DeviceCSR, rap
    A = DeviceCSR.from_host(G.stencil27(4))
    P = DeviceCSR.from_host(G.uniform_rows(5, 2, seed=1, m=60))  # P.m != A.n
    with pytest.raises(SpgemmError, match="INVALID_ARG"):
        rap(A, P, None, handle)
