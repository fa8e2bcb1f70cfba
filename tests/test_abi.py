"""CPU: the C-ABI library builds, loads, and exports every symbol that
include/spgemm.h declares (no GPU compute here)."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "spgemm.h").read_text()
    return sorted(set(re.findall(r"SPGEMM_API\s+[\w\s\*]+?\b(spgemm_\w+)\s*\(", text)))


def test_header_declarations_listed():
    names = declared_functions()
    assert "spgemm_csr_f64" in names and "spgemm_csr_f32" in names
    from gpuspgemm_b200 import _native
    assert set(names) == set(_native.SIGNATURES), set(names) ^ set(_native.SIGNATURES)


def test_library_exports_every_symbol(native_lib):
    for name in declared_functions():
        assert hasattr(native_lib, name), name


def test_status_strings_and_version(native_lib):
    from gpuspgemm_b200 import _native as N
    assert native_lib.spgemm_abi_version() == N.ABI_VERSION == 5
    assert native_lib.spgemm_status_string(0) == b"SPGEMM_OK"
    assert native_lib.spgemm_status_string(4) == b"SPGEMM_ERR_OVERFLOW"


def test_argument_errors_without_gpu(native_lib):
    from gpuspgemm_b200 import _native as N
    # NULL handle is rejected on the host before any CUDA call
    out = N.CsrOut()
    a = N.CsrView(2, 2, 0, None, None, None)
    st = native_lib.spgemm_csr_f64(None, C.byref(a), C.byref(a), C.byref(out), None)
    assert st == 1
    assert b"handle" in native_lib.spgemm_last_error_string()
    assert native_lib.spgemm_csr_free(None, None) == 0
    assert native_lib.spgemm_host_csr_free(None) == 0


def test_ladders_are_monotone(native_lib):
    from gpuspgemm_b200 import _native as N
    for which in (0, 1):
        for nbytes in (4, 8):
            nb = C.c_int()
            lim = (C.c_int64 * 16)()
            assert native_lib.spgemm_ladder_info(None, which, nbytes, C.byref(nb), lim) == 0
            vals = list(lim)[: nb.value]
            assert nb.value >= 5
            assert all(x <= y for x, y in zip(vals, vals[1:]))
            assert vals[-1] == 2**31 - 1


def test_esc_ladder_matches_bitmap_ladder(native_lib):
    """The one-pass ladder with expand-sort-compress team bins routes rows
    exactly like the bitmap ladder it replaces them in (same bins, same
    limits), so SPGEMM_OPT_ESC changes kernels, never the binning."""
    def limits(which, nbytes):
        nb = C.c_int()
        lim = (C.c_int64 * 16)()
        assert native_lib.spgemm_ladder_info(None, which, nbytes, C.byref(nb), lim) == 0
        return list(lim)[: nb.value]
    for nbytes in (4, 8):
        assert limits(4, nbytes) == limits(2, nbytes)
        assert limits(4, nbytes)[:4] == [12, 48, 192, 768]
    nb = C.c_int()
    lim = (C.c_int64 * 16)()
    assert native_lib.spgemm_ladder_info(None, 5, 8, C.byref(nb), lim) != 0
