"""GPU: the library against the REFERENCE's own GPU code on the same inputs.

oracle/_ref/libref_proposal.so is the reference's proposal_inner<T,
Parameters<CC80>> and its cuSPARSE-ALG2 validate path, compiled from the
reference sources for sm_100a (`make -C oracle ref`).  These tests need that
build; they are skipped where it is absent.  Besides parity they time both
implementations the way the reference's `measure` lambda does (wall clock
around the call plus a device synchronize, C allocated and freed inside;
src/apps/proposal.cu:28-35) and, when SPGEMM_PARITY_OUT names a folder, write
the figures to ref_compare.json there.
"""
import json
import os
import time
from pathlib import Path

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G

pytestmark = pytest.mark.gpu

OUT = Path(os.environ["SPGEMM_PARITY_OUT"]) if os.environ.get("SPGEMM_PARITY_OUT") else None
RECORDS = {}


@pytest.fixture(scope="module", autouse=True)
def _dump():
    yield
    if OUT is not None and OUT.is_dir() and RECORDS:
        (OUT / "ref_compare.json").write_text(json.dumps(RECORDS, indent=1))


def _ours_times(A, dtype, handle, warmups=3, runs=5):
    import torch

    from gpuspgemm_b200.api import DeviceCSR, proposal
    dA = DeviceCSR.from_host(A.astype(dtype))
    for _ in range(warmups):
        C = proposal(dA, dA, handle)
        del C
    ts = []
    for _ in range(runs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        C = proposal(dA, dA, handle)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)  # the clock stops before C is freed
        del C
    C = proposal(dA, dA, handle).to_host()
    return ts, C


CASES = {
    "uniform4096x8_f64": (lambda: G.uniform_rows(4096, 8), np.float64),
    "powerlaw1M_f64": (lambda: G.power_law(), np.float64),
    "powerlaw1M_f32": (lambda: G.power_law(), np.float32),
    # the power-law matrix at ~3.1 M nnz (Zipf exponent 2.2)
    "powerlaw1M_zipf2.2_f64": (lambda: G.power_law(1_000_000, 2.2, 4700), np.float64),
}


def _reference_equal(C, R):
    """The reference's operator== (csr.cuh:218-239): same structure, every
    value within 1e-8 + 1e-5 * max(|l|, |r|)."""
    if not (np.array_equal(C.rpt, R.rpt) and np.array_equal(C.col, R.col)):
        return False
    l, r = C.val.astype(np.float64), R.val.astype(np.float64)
    return bool(np.all(np.abs(l - r) <= 1e-8 + 1e-5 * np.maximum(np.abs(l), np.abs(r))))


@pytest.mark.parametrize("name", list(CASES))
def test_against_reference_build(handle, oracle_mod, name):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    make, dt = CASES[name]
    A = make().astype(dt)
    R = oracle_mod.ref_proposal(A, A, dt)
    ts, C = _ours_times(A, dt, handle)
    assert np.array_equal(C.rpt, R.rpt), "row pointers differ from the reference"
    assert np.array_equal(C.col, R.col), "column indices differ from the reference"
    rel = np.abs(C.val.astype(np.float64) - R.val.astype(np.float64))
    denom = np.abs(R.val.astype(np.float64))
    nz = denom > 0
    max_rel = float((rel[nz] / denom[nz]).max()) if np.any(nz) else 0.0
    tol = 1e-12 if dt == np.float64 else 1e-5
    assert max_rel <= tol, max_rel
    ref_ts, nip = oracle_mod.ref_time("proposal", A, A, dt, warmups=3, runs=5)
    rec = {"nip": nip, "nnz_C": int(C.nnz), "max_rel_vs_reference": max_rel,
           "ours_s": ts, "reference_proposal_s": ref_ts,
           "ours_gflops_median": 2 * nip / float(np.median(ts)) / 1e9,
           "reference_gflops_median": 2 * nip / float(np.median(ref_ts)) / 1e9}
    # the reference's validate path (cuSPARSE SpGEMM ALG2, common.hpp:109-126):
    # identical structure, values within its own tolerance
    CS = oracle_mod.ref_cusparse2(A, A, dt)
    assert np.array_equal(C.rpt, CS.rpt), "row pointers differ from cuSPARSE ALG2"
    assert np.array_equal(C.col, CS.col), "column indices differ from cuSPARSE ALG2"
    assert _reference_equal(C, CS)
    # each sums the products in its own order: compare against the
    # cancellation-aware bound sum_k |a_ik||b_kj| (the relative error where
    # the values cannot cancel)
    A64 = A.astype(np.float64)
    bound = oracle_mod.abs_bound(A64, A64, CS)
    diff = np.abs(C.val.astype(np.float64) - CS.val.astype(np.float64))
    max_cond_cs = float((diff / np.where(bound > 0, bound, 1.0)).max()) if CS.nnz else 0.0
    assert max_cond_cs <= tol, max_cond_cs
    rec["max_err_over_bound_vs_cusparse2"] = max_cond_cs
    del CS
    try:
        cs_ts, _ = oracle_mod.ref_time("cusparse2", A, A, dt, warmups=1, runs=3)
        rec["cusparse2_s"] = cs_ts
        rec["cusparse2_gflops_median"] = 2 * nip / float(np.median(cs_ts)) / 1e9
    except Exception as e:  # the reference records failed cuSPARSE runs as 0
        rec["cusparse2_error"] = str(e)
    # the vendored OpSparse last: its runs slowed the proposal timed after them
    if oracle_mod.ops_available(dt):
        O = oracle_mod.ops_run(A, A, dt)
        rec["opsparse_structure_equal"] = bool(np.array_equal(O.rpt, C.rpt)
                                               and np.array_equal(O.col, C.col))
        ops_ts = oracle_mod.ops_time(A, A, dt, warmups=2, runs=3)
        rec["opsparse_s"] = ops_ts
        rec["opsparse_gflops_median"] = 2 * nip / float(np.median(ops_ts)) / 1e9
        assert rec["opsparse_structure_equal"]
    RECORDS[name] = rec


def test_galerkin_against_reference_build(handle, oracle_mod):
    """R * (A * P) on the 27-point stencil of 60^3: the reference runs it as
    two proposal calls with a host transpose between them; the library as one
    chained call (R = P^T transposed on the device)."""
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    import torch

    from gpuspgemm_b200.api import DeviceCSR, rap
    A = G.stencil27(60)
    P = G.aggregation_prolongator(60, seed=5)
    R = oracle_mod.transpose(P)
    AP_ref = oracle_mod.ref_proposal(A, P, np.float64)
    C_ref = oracle_mod.ref_proposal(R, AP_ref, np.float64)
    dA, dP = DeviceCSR.from_host(A), DeviceCSR.from_host(P)
    for _ in range(3):
        del_c = rap(dA, dP, None, handle)
        del del_c
    ts = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        C = rap(dA, dP, None, handle)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)  # the clock stops before C is freed
        if len(ts) < 5:
            del C
    C = C.to_host()
    assert np.array_equal(C.rpt, C_ref.rpt) and np.array_equal(C.col, C_ref.col)
    # the stencil's rows sum to zero: compare against the magnitude bound
    absd = lambda M: type(M)(M.m, M.n, M.rpt, M.col, np.abs(M.val))  # noqa: E731
    bound = oracle_mod.spgemm(absd(R), oracle_mod.spgemm(absd(A), absd(P)))
    err = float((np.abs(C.val - C_ref.val) / bound.val).max())
    assert err <= 1e-12, err
    t_ap, nip_ap = oracle_mod.ref_time("proposal", A, P, np.float64, warmups=3, runs=5)
    t_rap, nip_rap = oracle_mod.ref_time("proposal", R, AP_ref, np.float64, warmups=3, runs=5)
    ref_chain = float(np.median(t_ap)) + float(np.median(t_rap))
    nip = nip_ap + nip_rap
    RECORDS["galerkin60_f64"] = {
        "nip": nip, "nnz_C": int(C.nnz), "max_err_vs_reference_over_bound": err,
        "ours_chain_s": ts, "reference_AP_s": t_ap, "reference_RAP_s": t_rap,
        "ours_gflops_median": 2 * nip / float(np.median(ts)) / 1e9,
        "reference_gflops_median_two_calls": 2 * nip / ref_chain / 1e9,
        "note": "reference time excludes its host transpose of P",
    }
