"""CPU: the oracle against a pure-Python restatement and against the golden
vectors produced by the reference's own GPU code (tests/golden/)."""
import json
from pathlib import Path

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR, load_csr

GOLDEN = Path(__file__).resolve().parent / "golden"


def py_gustavson(A: HostCSR, B: HostCSR):
    """Slow dict-based C = A*B in FP64, products summed in A-row order."""
    rpt = [0]
    cols, vals = [], []
    for i in range(A.m):
        acc = {}
        for p in range(A.rpt[i], A.rpt[i + 1]):
            k = A.col[p]
            a = float(A.val[p])
            for q in range(B.rpt[k], B.rpt[k + 1]):
                j = int(B.col[q])
                acc[j] = acc.get(j, 0.0) + a * float(B.val[q])
        for j in sorted(acc):
            cols.append(j)
            vals.append(acc[j])
        rpt.append(len(cols))
    return HostCSR(A.m, B.n, np.array(rpt, np.int32), np.array(cols, np.int32),
                   np.array(vals, np.float64))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_python(oracle_mod, seed):
    A = G.uniform_rows(60, 5, seed=seed, m=40)
    B = G.uniform_rows(70, 4, seed=seed + 100, m=60)
    C = oracle_mod.spgemm(A, B)
    R = py_gustavson(A, B)
    assert np.array_equal(C.rpt, R.rpt)
    assert np.array_equal(C.col, R.col)
    # same summation order and rounding -> bit-identical
    assert np.array_equal(C.val, R.val)


def test_oracle_keeps_cancelled_entries(oracle_mod):
    # [[1, 1], [0, 0]] @ [[1], [-1]] has a structural entry whose value is 0
    A = HostCSR(2, 2, np.array([0, 2, 2], np.int32), np.array([0, 1], np.int32),
                np.array([1.0, 1.0]))
    B = HostCSR(2, 1, np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32),
                np.array([1.0, -1.0]))
    C = oracle_mod.spgemm(A, B)
    assert C.nnz == 1 and C.col.tolist() == [0] and C.val.tolist() == [0.0]


def test_oracle_powerlaw_matches_python(oracle_mod):
    A = G.power_law(400, 2.0, 60, seed=5)
    C = oracle_mod.spgemm(A, A)
    R = py_gustavson(A, A)
    assert np.array_equal(C.rpt, R.rpt) and np.array_equal(C.col, R.col)
    assert np.array_equal(C.val, R.val)
    assert oracle_mod.nip(A, A) == int(sum(
        A.rpt[c + 1] - A.rpt[c] for c in A.col))


def test_oracle_f32_accumulates_in_f32(oracle_mod):
    A = G.uniform_rows(80, 6, seed=9).astype(np.float32)
    C = oracle_mod.spgemm(A, A)
    assert C.val.dtype == np.float32
    R = py_gustavson(A.astype(np.float64), A.astype(np.float64))
    assert np.array_equal(C.col, R.col)
    assert np.max(np.abs(C.val - R.val)) < 1e-5


def test_compare_reports_errors(oracle_mod):
    A = G.uniform_rows(50, 4, seed=3)
    C = oracle_mod.spgemm(A, A)
    D = HostCSR(C.m, C.n, C.rpt.copy(), C.col.copy(), C.val.copy())
    D.val[0] *= 1 + 1e-9
    r = oracle_mod.compare(D, C, oracle_mod.abs_bound(A, A, C))
    assert r["col_equal"] and not r["bit_exact"]
    assert 5e-10 < r["max_rel"] < 2e-9
    assert r["ref_mismatch"] == 0


def _golden_cases():
    man = GOLDEN / "manifest.json"
    if not man.exists():
        return []
    return sorted(json.loads(man.read_text()).items())


@pytest.mark.parametrize("name,entry", _golden_cases() or [pytest.param(
    None, None, marks=pytest.mark.skip(reason="golden vectors not generated"))])
def test_oracle_against_reference_golden(oracle_mod, name, entry):
    dt = np.dtype(entry["dtype"])
    A = load_csr(GOLDEN / f"{name}.A.csr", dt)
    B = load_csr(GOLDEN / f"{name}.B.csr", dt)
    C = oracle_mod.spgemm(A, B, dt)
    assert oracle_mod.nip(A, B) == entry["nip"]
    bound = oracle_mod.abs_bound(A, B, C)
    for which in ("proposal", "cusparse2"):
        path = GOLDEN / f"{name}.C_{which}.csr"
        if not path.exists():
            continue
        R = load_csr(path, dt)
        res = oracle_mod.compare(R, C, bound)
        assert res["rpt_equal"] and res["col_equal"], (which, res)
        tol = 1e-12 if dt == np.float64 else 1e-5
        # condition-aware bound: |dc| <= tol * sum_k |a_ik||b_kj|
        assert res.get("max_cond", 0.0) <= tol, (which, res)


def test_oracle_transpose_matches_scipy():
    """The oracle's transpose (stable counting sort) against scipy's."""
    import scipy.sparse as sp

    import oracle
    from gpuspgemm_b200 import generators as G
    for A in (G.power_law(3000, 2.0, 300, seed=3), G.uniform_rows(40, 3, seed=3, m=500),
              G.aggregation_prolongator(9)):
        T = oracle.transpose(A)
        S = sp.csr_matrix((A.val, A.col, A.rpt), shape=(A.m, A.n)).T.tocsr()
        S.sort_indices()
        assert (T.m, T.n) == S.shape
        assert np.array_equal(T.rpt, S.indptr) and np.array_equal(T.col, S.indices)
        assert np.array_equal(T.val, S.data)
        G2 = G.transpose(A)
        assert np.array_equal(T.col, G2.col) and np.array_equal(T.val, G2.val)
