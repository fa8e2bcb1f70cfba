"""GPU: plans -- the product's structure computed once, its fill phase replayed
as one CUDA graph after the operands' values change in place.  Every replay
is checked against the oracle on the new values (structure bit-exact, values
within the FP64/FP32 tolerances of the parity tests)."""
import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float64): 1e-12, np.dtype(np.float32): 1e-5}


def _check(oracle_mod, A, B, C, dtype):
    dtype = np.dtype(dtype)
    A64 = A.astype(dtype).astype(np.float64)
    B64 = B.astype(dtype).astype(np.float64)
    R = oracle_mod.spgemm(A64, B64, np.float64)
    res = oracle_mod.compare(C, R, oracle_mod.abs_bound(A64, B64, R))
    assert res["rpt_equal"] and res["col_equal"], res
    assert res["max_cond"] <= TOL[dtype], res


def _revalue(dA, A, seed):
    """New values for A, written in place into the device array the plan reads."""
    import torch
    vals = np.random.default_rng(seed).uniform(-1, 1, A.nnz)
    dA.val.copy_(torch.from_numpy(vals.astype(A.val.dtype)))
    return HostCSR(A.m, A.n, A.rpt, A.col, vals.astype(A.val.dtype))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_plan_replays_new_values(handle, oracle_mod, dtype):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, plan
    A = G.power_law(30000, 2.0, 3000, seed=21).astype(dtype)
    B = G.power_law(30000, 2.0, 3000, seed=22).astype(dtype)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    p = plan(dA, dB, handle=handle)
    try:
        _check(oracle_mod, A, B, p.result.to_host(), dtype)
        for k in range(3):
            A = _revalue(dA, A, 100 + k)
            p.execute()
            torch.cuda.synchronize()
            _check(oracle_mod, A, B, p.result.to_host(), dtype)
        p.check()
        assert p.info()["candidates"] == [p.info()["candidates"][0]]
    finally:
        p.close()


def test_plan_tuned(handle, oracle_mod):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, plan
    A = G.power_law(50000, 2.0, 2000, seed=31)
    dA = DeviceCSR.from_host(A)
    p = plan(dA, dA, tune=True, handle=handle)
    try:
        info = p.info()
        # team limits x {1, 0.75, 0.5}, CTA limits x {1, 0.5}, 4 or 8 streams
        assert len(info["candidates"]) == 12 and 0 <= info["chosen"] < 12
        assert {(c["team_scale"], c["cta_scale"], c["streams"]) for c in info["candidates"]} == \
            {(t, c, s) for t in (1.0, 0.75, 0.5) for c in (1.0, 0.5) for s in (4, 8)}
        assert all(c["ms"] > 0 for c in info["candidates"])
        best = info["candidates"][info["chosen"]]["ms"]
        assert best == min(c["ms"] for c in info["candidates"])
        _check(oracle_mod, A, A, p.result.to_host(), np.float64)
        A2 = _revalue(dA, A, 7)
        p.execute()
        torch.cuda.synchronize()
        _check(oracle_mod, A2, A2, p.result.to_host(), np.float64)
        p.check()
    finally:
        p.close()


def test_plan_batch(handle, oracle_mod):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, pack_batch, plan_batch
    mats = [G._poisson_square(int(n), 10.0, 50 + i, np.float64)
            for i, n in enumerate([300, 1200, 4000, 64, 9000, 2500])]
    dev = [DeviceCSR.from_host(M) for M in mats]
    pb = pack_batch([(d, d) for d in dev])
    p = plan_batch(pb, tune=True, handle=handle)
    try:
        assert len(p.result) == len(mats)
        for M, c in zip(mats, p.result):
            _check(oracle_mod, M, M, c.to_host(), np.float64)
        # new values for the packed A (the plan reads pb.A's value array)
        rng = np.random.default_rng(9)
        new = rng.uniform(-1, 1, pb.A.nnz)
        pb.A.val.copy_(torch.from_numpy(new))
        p.execute()
        torch.cuda.synchronize()
        off = 0
        for M, c in zip(mats, p.result):
            Mn = HostCSR(M.m, M.n, M.rpt, M.col, new[off:off + M.nnz])
            off += M.nnz
            _check(oracle_mod, Mn, M, c.to_host(), np.float64)
        p.check()
    finally:
        p.close()


def test_plan_heavy_row_global_bin(handle, oracle_mod):
    """A row in the global bitmap bin: the plan owns the bitmaps it replays on."""
    import torch

    from gpuspgemm_b200.api import DeviceCSR, plan
    rng = np.random.default_rng(51)
    B = G.uniform_rows(300_000, 300, seed=52, m=1000)
    A = HostCSR(3, 1000, np.array([0, 1000, 1000, 1003], np.int32),
                np.concatenate([np.arange(1000, dtype=np.int32), np.array([1, 5, 9], np.int32)]),
                rng.uniform(0.1, 1.0, 1003))
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    p = plan(dA, dB, handle=handle)
    try:
        A2 = _revalue(dA, A, 3)
        p.execute()
        p.execute()
        torch.cuda.synchronize()
        _check(oracle_mod, A2, B, p.result.to_host(), np.float64)
        p.check()
    finally:
        p.close()


def test_plan_empty_product(handle):
    from gpuspgemm_b200.api import DeviceCSR, plan
    A = HostCSR(4, 3, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = G.uniform_rows(5, 2, seed=1, m=3)
    p = plan(DeviceCSR.from_host(A), DeviceCSR.from_host(B), handle=handle)
    try:
        p.execute()  # nothing to recompute
        p.check()
        assert p.result.nnz == 0
    finally:
        p.close()
