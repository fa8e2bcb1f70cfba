"""CPU: the bounds of the cluster count bin's insert loop.

tests/cluster_probe_host.cpp compiles the kernel's own insert step
(gpuspgemm_b200/csrc/cluster_insert.cuh) against a plain array that stands in
for the cluster's distributed shared memory, with the table size of the
library's cluster bin (4 CTAs x 55,296 slots, slices of 1,024 A entries).
A row whose distinct keys exceed the table must spill (go to the global bin)
with every key probing a bounded number of slots; rows that fit must count
exactly.
"""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
SRC = HERE / "cluster_probe_host.cpp"
T, CSIZE, THREADS = 55296, 4, 1024


@pytest.fixture(scope="module")
def probe_bin(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("probe") / "cluster_probe_host"
    subprocess.run([cxx, "-O2", "-std=c++17", str(SRC), "-o", str(out)], check=True)
    return out


def run(probe_bin, case):
    res = subprocess.run([str(probe_bin), case, str(T), str(CSIZE), str(THREADS)],
                         capture_output=True, text=True, check=True, timeout=120)
    return json.loads(res.stdout)


def test_slice_past_the_table_spills_with_bounded_probes(probe_bin):
    r = run(probe_bin, "overflow")
    assert r["distinct"] > r["slots"]          # one slice holds more keys than the table
    assert r["spilled"] == 1                   # the row goes to the fail list
    assert r["max_probes"] <= r["max_probes_allowed"]
    # the table stops filling near its load limit, well short of full
    assert r["occupied"] <= r["limit"] + CSIZE * 256
    assert r["occupied"] < r["slots"]
    assert r["keys_after_spill"] > 0 and r["probes_after_spill"] == 0


def test_rows_that_fit_count_exactly(probe_bin):
    for case in ("fits", "repeats"):
        r = run(probe_bin, case)
        assert r["spilled"] == 0, (case, r)
        assert r["count"] == r["distinct"], (case, r)
        assert r["occupied"] == r["distinct"], (case, r)
        assert r["max_probes"] <= r["max_probes_allowed"], (case, r)


def test_long_probe_chain_spills_at_the_cap(probe_bin):
    r = run(probe_bin, "chain")
    assert r["spilled"] == 1
    assert r["max_probes"] == r["max_probes_allowed"]
    assert r["occupied"] <= r["max_probes_allowed"]
