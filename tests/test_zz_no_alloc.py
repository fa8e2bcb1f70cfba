"""GPU: the allocation-free row-size entry point, spgemm_row_nnz_noalloc.

It exists for callers that cannot allocate device memory where they size a
product (all memory already handed to their own pool, or an allocation there
would synchronise the device).  It must give exactly the row sizes of C -- the
differences of the oracle's row pointer, and of C.rpt from spgemm_csr_f64 --
and keep doing so on the next calls, since every call reuses the same fixed
scratch area.  The file name sorts last so that a run stopping at its first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def _view(d):
    from gpuspgemm_b200 import _native as N
    return N.CsrView(d.m, d.n, d.nnz, d.rpt.data_ptr(), d.col.data_ptr() if d.nnz else None,
                     d.val.data_ptr() if d.nnz else None)


def _noalloc_row_nnz(dA, dB):
    import torch

    from gpuspgemm_b200 import _native as N
    out = torch.full((dA.m,), -7, dtype=torch.int32, device=dA.rpt.device)
    va, vb = _view(dA), _view(dB)
    st = N.lib().spgemm_row_nnz_noalloc(C.byref(va), C.byref(vb), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _heavy_rows():
    """Rows of 3,000 and 1,500 A entries (several 1,024-entry chunks, ~10^5
    products each), empty rows in A and in B, and B.n close to 2^20."""
    rng = np.random.default_rng(84)
    B = G.uniform_rows((1 << 20) - 3, 40, seed=85, m=4000)
    b_rpt = B.rpt.copy()
    for r in (7, 1234, 3999):              # empty rows of B
        b_rpt[r + 1:] -= b_rpt[r + 1] - b_rpt[r]
    keep = np.ones(B.nnz, bool)
    for r in (7, 1234, 3999):
        keep[B.rpt[r]:B.rpt[r + 1]] = False
    B = HostCSR(B.m, B.n, b_rpt, B.col[keep], B.val[keep])
    rows = [np.sort(rng.choice(4000, 3000, replace=False)), np.array([], np.int64),
            np.sort(rng.choice(4000, 1500, replace=False)), np.array([7, 1234]),
            np.array([], np.int64), np.sort(rng.choice(4000, 17, replace=False))]
    rpt = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    col = np.concatenate(rows).astype(np.int32)
    A = HostCSR(len(rows), 4000, rpt, col, rng.uniform(-1, 1, col.size))
    return A, B


@pytest.mark.parametrize("make", [
    lambda: (G.uniform_rows(4096, 8),) * 2,
    lambda: (G.power_law(20000, 2.0, 1000, seed=81),) * 2,
    lambda: (G.uniform_rows(900, 7, seed=82, m=300), G.uniform_rows(5000, 9, seed=83, m=900)),
    _heavy_rows,
], ids=["uniform4096", "powerlaw20k", "rect", "heavy_empty_wide"])
def test_noalloc_row_nnz_matches_product(make, oracle_mod):
    from gpuspgemm_b200.api import DeviceCSR, Handle, proposal
    A, B = make()
    oracle_nnz = np.diff(oracle_mod.spgemm(A, B, np.float64).rpt)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    h = Handle()
    try:
        expect = np.diff(proposal(dA, dB, h).rpt.cpu().numpy())
    finally:
        h.close()
    assert np.array_equal(expect, oracle_nnz)
    for _ in range(3):  # the same scratch area, left by the call before
        got = _noalloc_row_nnz(dA, dB)
        assert np.array_equal(got, oracle_nnz)


def test_noalloc_flags_rows_with_out_of_range_columns(oracle_mod):
    """A column of B at or past B.n is skipped (it would index outside the
    scratch slot) and the rows of C that reach it report -1; the next call on
    valid operands is exact again."""
    from gpuspgemm_b200.api import DeviceCSR
    B = HostCSR(3, 64, np.array([0, 2, 4, 5], np.int32), np.array([1, 9, 3, 70, 5], np.int32),
                np.ones(5))
    A = HostCSR(3, 3, np.array([0, 1, 2, 4], np.int32), np.array([0, 1, 0, 2], np.int32),
                np.ones(4))
    got = _noalloc_row_nnz(DeviceCSR.from_host(A), DeviceCSR.from_host(B))
    assert got.tolist() == [2, -1, 3]
    U = G.uniform_rows(512, 6, seed=86)
    dU = DeviceCSR.from_host(U)
    ref = np.diff(oracle_mod.spgemm(U, U, np.float64).rpt)
    assert np.array_equal(_noalloc_row_nnz(dU, dU), ref)


def test_noalloc_rejects_too_many_columns():
    from gpuspgemm_b200 import _native as N
    A = N.CsrView(1, 4, 0, None, None, None)
    B = N.CsrView(4, (1 << 20) + 1, 0, None, None, None)
    st = N.lib().spgemm_row_nnz_noalloc(C.byref(A), C.byref(B), None, None)
    assert st == 1
    assert b"exceeds the allocation-free limit" in N.lib().spgemm_last_error_string()
