"""GPU: the allocation-free row-size entry point, spgemm_row_nnz_noalloc.

It exists for callers that cannot allocate device memory where they size a
product (all memory already handed to their own pool, or an allocation there
would synchronise the device).  It must give exactly the row sizes that the
regular product gives -- the differences of C.rpt from spgemm_csr_f64 -- and
keep doing so on the next call, since every call reuses the same fixed scratch
area.  The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G

pytestmark = pytest.mark.gpu


def _view(d):
    from gpuspgemm_b200 import _native as N
    return N.CsrView(d.m, d.n, d.nnz, d.rpt.data_ptr(), d.col.data_ptr() if d.nnz else None,
                     d.val.data_ptr() if d.nnz else None)


def _noalloc_row_nnz(dA, dB):
    import torch

    from gpuspgemm_b200 import _native as N
    out = torch.full((dA.m,), -1, dtype=torch.int32, device=dA.rpt.device)
    va, vb = _view(dA), _view(dB)
    st = N.lib().spgemm_row_nnz_noalloc(C.byref(va), C.byref(vb), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("make", [
    lambda: (G.uniform_rows(4096, 8),) * 2,
    lambda: (G.power_law(20000, 2.0, 1000, seed=81),) * 2,
    lambda: (G.uniform_rows(900, 7, seed=82, m=300), G.uniform_rows(5000, 9, seed=83, m=900)),
])
def test_noalloc_row_nnz_matches_product(make):
    from gpuspgemm_b200.api import DeviceCSR, Handle, proposal
    A, B = make()
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    h = Handle()
    try:
        expect = np.diff(proposal(dA, dB, h).rpt.cpu().numpy())
    finally:
        h.close()
    first = _noalloc_row_nnz(dA, dB)
    second = _noalloc_row_nnz(dA, dB)  # same scratch area, left by the first call
    assert np.array_equal(first, expect)
    assert np.array_equal(second, expect)


def test_noalloc_rejects_too_many_columns():
    from gpuspgemm_b200 import _native as N
    A = N.CsrView(1, 4, 0, None, None, None)
    B = N.CsrView(4, (1 << 20) + 1, 0, None, None, None)
    st = N.lib().spgemm_row_nnz_noalloc(C.byref(A), C.byref(B), None, None)
    assert st == 1
    assert b"exceeds the allocation-free limit" in N.lib().spgemm_last_error_string()
