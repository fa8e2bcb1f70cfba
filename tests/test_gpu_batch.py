"""GPU: the batched form (spgemm_batch_*) -- many independent products run as
one binned product of block-diagonal operands.  Every product of the batch must
equal the same product run alone (structure bit-exact) and the CPU oracle
(values within tolerance)."""
import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def _host(d) -> HostCSR:
    return d.to_host()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_batch_matches_oracle_and_single_calls(handle, oracle_mod, dtype):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, batch, pack_batch, proposal
    pairs_h = list(G.batch_pairs(24, seed=91, dtype=dtype, rows_lo=16, rows_hi=2000))
    # rectangular and empty members too
    pairs_h.append((G.uniform_rows(300, 5, seed=92, m=120).astype(dtype),
                    G.uniform_rows(70, 4, seed=93, m=300).astype(dtype)))
    pairs_h.append((HostCSR(5, 3, np.zeros(6, np.int32), np.zeros(0, np.int32),
                            np.zeros(0, dtype)),
                    G.uniform_rows(4, 2, seed=94, m=3).astype(dtype)))
    pairs = [(DeviceCSR.from_host(a), DeviceCSR.from_host(b)) for a, b in pairs_h]
    pb = pack_batch(pairs)
    out = batch(pb, handle)
    assert len(out) == len(pairs)
    tol = 1e-12 if dtype == np.float64 else 1e-5
    for (a, b), (da, db), c in zip(pairs_h, pairs, out):
        ch = _host(c)
        assert (ch.m, ch.n) == (a.m, b.n)
        single = proposal(da, db, handle).to_host()
        assert np.array_equal(ch.rpt, single.rpt) and np.array_equal(ch.col, single.col)
        a64, b64 = a.astype(np.float64), b.astype(np.float64)
        R = oracle_mod.spgemm(a64, b64, np.float64)
        res = oracle_mod.compare(ch, R, oracle_mod.abs_bound(a64, b64, R))
        assert res["rpt_equal"] and res["col_equal"], res
        assert res.get("max_cond", 0.0) <= tol, res
    torch.cuda.synchronize()


def test_batch_packed_gpu_generator_and_groups(handle, oracle_mod):
    import torch

    from gpuspgemm_b200.api import PackedBatch, batch
    a_off, b_off, c_off, A, B = G.batch_packed_gpu(40, seed=95, rows_lo=64, rows_hi=3000)
    pb = PackedBatch(a_off, b_off, c_off, A, B)
    out = batch(pb, handle)
    Ah, Bh = A.to_host(), B.to_host()
    for i in (0, 7, 39):
        r0, r1 = int(a_off[i]), int(a_off[i + 1])
        # product i alone on the CPU, in local indices
        rpt = Ah.rpt[r0:r1 + 1] - Ah.rpt[r0]
        Ai = HostCSR(r1 - r0, r1 - r0, rpt, Ah.col[Ah.rpt[r0]:Ah.rpt[r1]] - r0,
                     Ah.val[Ah.rpt[r0]:Ah.rpt[r1]].astype(np.float64))
        rptb = Bh.rpt[r0:r1 + 1] - Bh.rpt[r0]
        Bi = HostCSR(r1 - r0, r1 - r0, rptb, Bh.col[Bh.rpt[r0]:Bh.rpt[r1]] - r0,
                     Bh.val[Bh.rpt[r0]:Bh.rpt[r1]].astype(np.float64))
        R = oracle_mod.spgemm(Ai, Bi, np.float64)
        ch = out[i].to_host()
        res = oracle_mod.compare(ch, R, oracle_mod.abs_bound(Ai, Bi, R))
        assert res["rpt_equal"] and res["col_equal"], res
        assert res["max_cond"] <= 1e-5, res
    assert handle._last_groups >= 1
    torch.cuda.synchronize()


def _packed_member(M, off, i):
    """Product i's square operand, in local indices, from a packed operand
    (device tensors sliced on the device, then copied)."""
    r0, r1 = int(off[i]), int(off[i + 1])
    rpt = M.rpt[r0:r1 + 1].cpu().numpy()
    s0, s1 = int(rpt[0]), int(rpt[-1])
    return HostCSR(r1 - r0, r1 - r0, (rpt - s0).astype(np.int32),
                   (M.col[s0:s1].cpu().numpy() - r0).astype(np.int32),
                   M.val[s0:s1].cpu().numpy().astype(np.float64))


def test_full_batched_workload_sampled_parity(handle, oracle_mod):
    """The batched workload at its stated size: 4,096 independent FP32
    products (rows log-uniform in [64, 16384], Poisson(U[6, 40]) nnz per row,
    ~6.8 G nonzeros of C) run as one batch; 48 products drawn at random, plus
    the largest and the smallest, checked against the oracle."""
    import torch

    from gpuspgemm_b200.api import PackedBatch, batch
    a_off, b_off, c_off, A, B = G.batch_packed_gpu(4096, seed=20261203, dtype=torch.float32)
    pb = PackedBatch(a_off, b_off, c_off, A, B)
    out = batch(pb, handle)
    assert len(out) == 4096
    assert sum(c.nnz for c in out) > 6_000_000_000
    sizes = np.diff(np.asarray(a_off))
    rng = np.random.default_rng(77)
    picks = set(rng.choice(4096, 48, replace=False).tolist())
    picks |= {int(np.argmax(sizes)), int(np.argmin(sizes))}
    for i in sorted(picks):
        Ai = _packed_member(A, a_off, i)
        Bi = _packed_member(B, b_off, i)
        R = oracle_mod.spgemm(Ai, Bi, np.float64)
        ch = out[i].to_host()
        res = oracle_mod.compare(ch, R, oracle_mod.abs_bound(Ai, Bi, R))
        assert res["rpt_equal"] and res["col_equal"], (i, res)
        assert res["max_cond"] <= 1e-5, (i, res)
    del out
    torch.cuda.synchronize()


def test_get_nip_many_matches_single_calls(handle, oracle_mod):
    """One-launch sizing of many pairs: empty A, a pair larger than one CTA's
    chunk (16384 A entries), rectangular pairs."""
    import numpy as np

    from gpuspgemm_b200 import generators as G
    from gpuspgemm_b200.api import DeviceCSR, get_nip, get_nip_many
    from gpuspgemm_b200.csr import HostCSR
    mats = [
        (G.uniform_rows(50, 3, seed=1, m=40), G.uniform_rows(70, 4, seed=2, m=50)),
        (HostCSR(5, 50, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)),
         G.uniform_rows(9, 2, seed=3, m=50)),
        (G.power_law(40000, 2.0, 800, seed=4),) * 2,
        (G.uniform_rows(300, 8, seed=5),) * 2,
    ]
    pairs = [(DeviceCSR.from_host(a), DeviceCSR.from_host(b)) for a, b in mats]
    got = get_nip_many(pairs, handle)
    assert got == [get_nip(a, b, handle) for a, b in pairs]
    assert got == [oracle_mod.nip(a, b) for a, b in mats]
    assert got[2] > 16384 and get_nip_many([], handle) == []
