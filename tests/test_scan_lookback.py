"""CPU: the one-pass row pointer's look-back scan (k_rpt_scan1) run on the host.

The kernel's own source (gpuspgemm_b200/csrc/k_bin.cu) is compiled against the
host SIMT emulation in tests/simt_host (one OS thread per CUDA thread, CTAs in
ticket order) and driven by tests/simt_host/scan_lookback_host.cpp:

* exact exclusive scans, totals and maxima for 1 to 74 tiles of 4,096 rows;
* the same with every tile's prefix withheld (only tile 0 publishes one), so
  each look-back adds tile sums back to tile 0 across several 32-tile windows;
* a predecessor whose ticket is taken but which never publishes: the wait
  ends after its bounded number of rounds and reports kStWait instead of
  spinning (the wait itself is never run on a GPU to see it end).

The two test knobs are patched into the generated copy only; the patterns they
replace are asserted, so a change to the kernel fails here loudly.
"""
import json
import re
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = ROOT / "gpuspgemm_b200" / "csrc"
SIM = HERE / "simt_host"
K_ST_WAIT = 64


def host_source() -> str:
    """k_bin.cu's kernels for the host emulation: each __shared__ variable
    becomes a reference into the emulated CTA's static memory."""
    src = (CSRC / "k_bin.cu").read_text()
    body = src[: src.index("cudaError_t launch_nip_hist")]
    out, off = [], 0
    for line in body.split("\n"):
        if "__global__" in line:
            off = 0
        arr = re.match(r"(\s*)__shared__ ([\w ]+?) (\w+)\[(.+)\];", line)
        one = re.match(r"(\s*)__shared__ ([\w ]+?) (\w+);", line)
        if arr:
            ind, ty, name, dim = arr.groups()
            out.append(f"{ind}auto& {name} = *reinterpret_cast<{ty}(*)[{dim}]>("
                       f"emu_static<unsigned char>() + {off});")
            off += 20000
        elif one:
            ind, ty, name = one.groups()
            out.append(f"{ind}auto& {name} = *reinterpret_cast<{ty}*>("
                       f"emu_static<unsigned char>() + {off});")
            off += 64
        else:
            out.append(line)
    body = "\n".join(out)
    assert off <= 262144
    spins = "constexpr int kLookbackSpins = 1 << 20;"
    assert body.count(spins) == 1, "the look-back's wait bound changed"
    body = body.replace(spins, "").replace("kLookbackSpins", "emu_lookback_spins")
    publish = "            if (tile > 0)\n                atomicExch(state + 1 + tile,"
    assert body.count(publish) == 1, "the look-back's prefix publication changed"
    body = body.replace(publish, "            if (tile > 0 && !emu_withhold_prefix)\n"
                                 "                atomicExch(state + 1 + tile,")
    body = body.replace('#include "cta.cuh"\n#include "kernels.hpp"\n', "")
    head = ('#include "cuda_emu.h"\n#include "kernels.hpp"\n'
            "inline bool emu_withhold_prefix = false;\n"
            "inline int emu_lookback_spins = 1 << 20;\n"
            '#include "common.cuh"\n#include "cta.cuh"\n')
    return head + body + "}  // namespace b200\n"


@pytest.fixture(scope="module")
def scan_bin(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("scan")
    (d / "k_bin_host.cpp").write_text(host_source())
    out = d / "scan_lookback_host"
    subprocess.run([cxx, "-std=c++20", "-O1", "-pthread", f"-I{d}", f"-I{SIM}",
                    f"-I{SIM / 'fake'}", f"-I{CSRC}", f"-I{ROOT / 'include'}",
                    str(SIM / "scan_lookback_host.cpp"), "-o", str(out)],
                   check=True, timeout=600)
    return out


def run(scan_bin, *args):
    res = subprocess.run([str(scan_bin), *args], capture_output=True, text=True, timeout=600)
    return res.returncode, [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]


@pytest.mark.parametrize("withhold", ["0", "1"])
def test_lookback_scan_is_exact(scan_bin, withhold):
    rc, cases = run(scan_bin, "scan", withhold)
    assert len(cases) == 8
    for c in cases:
        assert c["ok"], c
        assert c["wrong"] == 0 and c["total"] == c["want_total"] and c["max"] == c["want_max"]
    assert max(c["tiles"] for c in cases) == 74
    assert rc == 0


def test_lookback_wait_is_bounded(scan_bin):
    rc, cases = run(scan_bin, "wait")
    assert rc == 0 and len(cases) == 1
    c = cases[0]
    assert c["wait_flag"] == K_ST_WAIT
    assert c["status"] & K_ST_WAIT, c
    assert c["row"] == 1 and c["detail"] == 0  # tile 1 gave up on tile 0
