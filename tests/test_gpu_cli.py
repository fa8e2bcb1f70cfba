"""GPU: the reference-compatible CLI driver (gpuspgemm_b200/spgemm_app and
spgemm_app_f32) run as the reference's apps are run.

The reference's apps take `inputA inputB [--loglevel L] validate | save OUT |
benchmark [--runs N --warmups N --pause MS]` (src/apps/common.hpp:40-82) and
print "Validation succeeded" (common.hpp:123-126) and one line per timed run,
`Run %2d: <t>ns | <flops> FLOPS` (common.hpp:196-204), which tasks.py parses
with `Run\\s+(\\d+): (.+)ns [|] (\\d+[.]\\d*) FLOPS` (tasks.py:104-107).  The
inputs are the golden `.csr` files made by the reference's own build; `save`
must write C with the structure of the reference's saved C.
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gpuspgemm_b200.csr import load_csr

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
PKG = Path(__file__).resolve().parent.parent / "gpuspgemm_b200"
RUN_LINE = re.compile(r"Run\s+(\d+): (.+)ns [|] (\d+[.]\d*) FLOPS")  # tasks.py:104-107

CASES = [("spgemm_app", "uniform512_f64"), ("spgemm_app", "powerlaw3000_f64"),
         ("spgemm_app_f32", "powerlaw3000_f32"), ("spgemm_app", "empty_rows_f64"),
         ("spgemm_app", "rect300x500x200_f64")]


@pytest.fixture(scope="module")
def apps(native_lib):
    for name in ("spgemm_app", "spgemm_app_f32"):
        assert (PKG / name).exists(), f"{name} was not built"
    return PKG


def run_app(app, *args, timeout=300):
    return subprocess.run([str(app), *map(str, args)], capture_output=True, text=True,
                          timeout=timeout)


@pytest.mark.parametrize("app,case", CASES)
def test_validate_succeeds(apps, app, case):
    r = run_app(apps / app, GOLDEN / f"{case}.A.csr", GOLDEN / f"{case}.B.csr", "validate")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Validation succeeded" in r.stdout, r.stdout


@pytest.mark.parametrize("app,case", CASES)
def test_save_matches_reference_structure(apps, app, case, tmp_path):
    out = tmp_path / "C.csr"
    r = run_app(apps / app, GOLDEN / f"{case}.A.csr", GOLDEN / f"{case}.B.csr", "save", out)
    assert r.returncode == 0, r.stdout + r.stderr
    got = load_csr(out)
    ref = load_csr(GOLDEN / f"{case}.C_proposal.csr")
    assert (got.m, got.n, got.nnz) == (ref.m, ref.n, ref.nnz)
    assert np.array_equal(got.rpt, ref.rpt)
    assert np.array_equal(got.col, ref.col)
    # values: the reference's own equality tolerance (csr.cuh:233-237)
    tol = 1e-8 + 1e-5 * np.maximum(np.abs(got.val), np.abs(ref.val))
    assert np.all(np.abs(got.val - ref.val) <= tol)
    # the file layout itself: int32 nnz, m, n, rpt, col, float64 val
    assert out.stat().st_size == 12 + 4 * (ref.m + 1) + 4 * ref.nnz + 8 * ref.nnz


def test_benchmark_lines_parse_like_tasks_py(apps):
    case = "powerlaw3000_f64"
    r = run_app(apps / "spgemm_app", GOLDEN / f"{case}.A.csr", GOLDEN / f"{case}.B.csr",
                "benchmark", "--runs", 2, "--warmups", 1, "--pause", 0)
    assert r.returncode == 0, r.stdout + r.stderr
    runs = [RUN_LINE.search(line) for line in r.stdout.splitlines()]
    runs = [m for m in runs if m]
    assert [int(m.group(1)) for m in runs] == [1, 2], r.stdout
    for m in runs:
        assert int(m.group(2)) > 0 and float(m.group(3)) > 0.0


def test_missing_input_is_an_error(apps, tmp_path):
    r = run_app(apps / "spgemm_app", tmp_path / "nope.csr", GOLDEN / "uniform512_f64.B.csr",
                "validate")
    assert r.returncode != 0
    assert "File does not exist" in (r.stdout + r.stderr)
