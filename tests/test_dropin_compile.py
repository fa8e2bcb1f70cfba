"""CPU: the C++ drop-in (gpuspgemm_b200/csrc/b200_proposal.hpp) builds against
the reference's own CSR type.

The reference's apps call `proposal::proposal(d_a, d_b)` on
`utils::DeviceCSR<T>` (src/apps/proposal.cu:22-35).  The swap is one line per
call: `b200::proposal(d_a, d_b)`.  This test compiles exactly those two
lambdas, with the reference's `utils/csr.cuh` and the drop-in header, into a
shared object linked against libspgemm_b200.so, for double and float.  It
needs the reference checkout (GPUSPGEMM_REFERENCE) and nvcc; it is skipped
without them.
"""
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

TU = r"""
#include <utils/csr.cuh>

#include "b200_proposal.hpp"

template<typename ValueType>
utils::HostCSR<ValueType> run(const utils::DeviceCSR<ValueType>& d_a,
                              const utils::DeviceCSR<ValueType>& d_b) {
    return b200::proposal(d_a, d_b).template to<utils::Location::Host>();
}

template<typename ValueType>
long long measure(const utils::DeviceCSR<ValueType>& d_a, const utils::DeviceCSR<ValueType>& d_b) {
    auto c = b200::proposal(d_a, d_b);
    utils::device_sync();
    return static_cast<long long>(c.nnz) + b200::get_nip(d_a, d_b);
}

template utils::HostCSR<double> run<double>(const utils::DeviceCSR<double>&,
                                            const utils::DeviceCSR<double>&);
template utils::HostCSR<float> run<float>(const utils::DeviceCSR<float>&,
                                          const utils::DeviceCSR<float>&);
template long long measure<double>(const utils::DeviceCSR<double>&,
                                   const utils::DeviceCSR<double>&);
template long long measure<float>(const utils::DeviceCSR<float>&,
                                  const utils::DeviceCSR<float>&);
"""


def test_dropin_builds_against_reference_devicecsr(tmp_path):
    sys.path.insert(0, str(ROOT))
    import oracle
    from gpuspgemm_b200 import build
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    utils_inc = oracle.REF_SRC / "libutils" / "include"
    if not (utils_inc / "utils" / "csr.cuh").exists():
        pytest.skip("reference checkout not present")
    lib = build.build()
    import torch
    torch_inc = Path(torch.__file__).resolve().parent / "include"
    src = tmp_path / "dropin.cu"
    src.write_text(TU)
    out = tmp_path / "libdropin.so"
    cmd = [nvcc, "-std=c++20", "-O2", "-DFMT_HEADER_ONLY", "-DNVTX_DISABLE",
           "--expt-relaxed-constexpr", "--extended-lambda",
           "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           f"-I{ROOT / 'oracle' / 'ref' / 'shim'}", f"-I{utils_inc}", f"-I{torch_inc}",
           f"-I{ROOT / 'gpuspgemm_b200' / 'csrc'}", f"-I{ROOT / 'include'}",
           str(src), "-o", str(out), f"-L{lib.parent}", "-lspgemm_b200"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert out.exists()
