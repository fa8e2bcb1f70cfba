"""GPU: the served form.  Requests of different sizes arrive while others are
running; each result must be the same as the product run alone (structure
bit-exact, values within tolerance) -- in the mix and alone."""
import time

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix(handle, oracle_mod):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, proposal
    from gpuspgemm_b200.serve import SpgemmServer, latency_summary
    rng = np.random.default_rng(101)
    mats = []
    for i in range(30):
        kind = rng.choice(3, p=[0.7, 0.25, 0.05])
        if kind == 0:
            A = G._poisson_square(int(rng.integers(200, 4000)), 12.0, 1000 + i, np.float64)
        elif kind == 1:
            A = G.power_law(int(rng.integers(20_000, 60_000)), 2.0, 600, seed=2000 + i)
        else:
            A = G.power_law(150_000, 2.0, 2000, seed=3000 + i)
        mats.append(A)
    dev = [DeviceCSR.from_host(A) for A in mats]
    alone = [proposal(d, d, handle).to_host() for d in dev]
    server = SpgemmServer(memory_budget=256 << 20, max_batch=8, workers=2)
    try:
        reqs = []
        # a few early arrivals, then bursts that arrive while those are running
        for k, d in enumerate(dev):
            reqs.append(server.submit(d, d))
            if k in (1, 12):
                time.sleep(0.002)
        for r in reqs:
            assert r.done.wait(timeout=120)
            assert r.error is None, r.error
    finally:
        server.close()
    for A, r, ref in zip(mats, reqs, alone):
        c = r.result.to_host()
        assert np.array_equal(c.rpt, ref.rpt) and np.array_equal(c.col, ref.col)
        R = oracle_mod.spgemm(A, A)
        res = oracle_mod.compare(c, R, oracle_mod.abs_bound(A, A, R))
        assert res["col_equal"] and res["max_rel"] <= 1e-12, res
    s = latency_summary(reqs)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    assert server.batches < len(reqs), "requests were never batched together"
    torch.cuda.synchronize()


def test_admission_respects_budget(handle):
    from gpuspgemm_b200.api import DeviceCSR
    from gpuspgemm_b200.serve import SpgemmServer
    A = DeviceCSR.from_host(G._poisson_square(3000, 12.0, 7, np.float64))
    server = SpgemmServer(memory_budget=1, max_batch=64, workers=1)  # every request alone
    try:
        reqs = [server.submit(A, A) for _ in range(6)]
        for r in reqs:
            assert r.done.wait(timeout=60) and r.error is None
    finally:
        server.close()
    assert server.batches == 6
