"""Host logic of the batched form: packing products into block-diagonal
operands (torch ops on whatever device the operands live on; CPU here)."""
import numpy as np
import pytest
import scipy.sparse as sp

from gpuspgemm_b200 import generators as G


def _dev(M):
    import torch

    from gpuspgemm_b200.api import DeviceCSR
    return DeviceCSR(M.m, M.n, torch.from_numpy(M.rpt.copy()), torch.from_numpy(M.col.copy()),
                     torch.from_numpy(M.val.copy()))


def _sp(M):
    return sp.csr_matrix((M.val, M.col, M.rpt), shape=(M.m, M.n))


def test_pack_matches_block_diag():
    from gpuspgemm_b200.api import pack_batch
    As = [G.power_law(300 + 50 * i, 2.0, 30, seed=i) for i in range(5)]
    As.append(G.uniform_rows(7, 2, seed=20, m=0))          # no rows
    As.append(G.uniform_rows(9, 0, seed=21, m=4))          # rows, no entries
    Bs = [G.uniform_rows(70 + i, 3, seed=10 + i, m=A.n) for i, A in enumerate(As)]
    pb = pack_batch([(_dev(a), _dev(b)) for a, b in zip(As, Bs)])
    RA = sp.block_diag([_sp(M) for M in As], format="csr")
    RB = sp.block_diag([_sp(M) for M in Bs], format="csr")
    for got, ref in ((pb.A, RA), (pb.B, RB)):
        assert (got.m, got.n) == ref.shape
        assert got.rpt.dtype == got.col.dtype
        assert np.array_equal(got.rpt.numpy(), ref.indptr)
        assert np.array_equal(got.col.numpy(), ref.indices)
        assert np.array_equal(got.val.numpy(), ref.data)
    assert pb.a_row_off.tolist() == list(np.cumsum([0] + [a.m for a in As]))
    assert pb.c_col_off.tolist() == list(np.cumsum([0] + [b.n for b in Bs]))


def test_pack_rejects_bad_pairs():
    from gpuspgemm_b200.api import pack_batch
    A = G.uniform_rows(5, 2, seed=1, m=3)
    B = G.uniform_rows(4, 2, seed=2, m=6)
    with pytest.raises(ValueError):
        pack_batch([(_dev(A), _dev(B))])
    with pytest.raises(ValueError):
        pack_batch([])


def test_pack_square_self_products_once():
    """C_i = A_i * A_i with square A_i, share=True: the packed B is the packed A
    itself, equal to the block diagonal of the A_i; without share (the
    default: a plan may update the packed values) or with distinct operands B
    is packed on its own."""
    from gpuspgemm_b200.api import pack_batch
    As = [G.power_law(200 + 40 * i, 2.0, 20, seed=30 + i) for i in range(4)]
    ds = [_dev(a) for a in As]
    assert pack_batch([(d, d) for d in ds]).B is not pack_batch([(d, d) for d in ds]).A
    pb = pack_batch([(d, d) for d in ds], share=True)
    assert pb.B is pb.A
    R = sp.block_diag([_sp(M) for M in As], format="csr")
    assert np.array_equal(pb.B.rpt.numpy(), R.indptr)
    assert np.array_equal(pb.B.col.numpy(), R.indices)
    # the same operands given as distinct objects: packed twice, same arrays
    pb2 = pack_batch([(d, _dev(a)) for d, a in zip(ds, As)], share=True)
    assert pb2.B is not pb2.A
    assert np.array_equal(pb2.B.col.numpy(), pb.A.col.numpy())
    # a rectangular A_i: B keeps its own column shifts
    Rt = G.uniform_rows(30, 3, seed=5, m=20)
    d = _dev(Rt)
    with pytest.raises(ValueError):
        pack_batch([(d, d)])  # 20 x 30 times 20 x 30 does not chain
