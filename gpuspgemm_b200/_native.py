"""ctypes binding of the C ABI in ``include/spgemm.h`` (libspgemm_b200.so).

Import fails loudly when the library has not been built: there is no CPU or
PyTorch fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libspgemm_b200.so"

SPGEMM_OK = 0
STATUS_NAMES = {
    0: "SPGEMM_OK",
    1: "SPGEMM_ERR_INVALID_ARG",
    2: "SPGEMM_ERR_OOM",
    3: "SPGEMM_ERR_UNSUPPORTED_DEVICE",
    4: "SPGEMM_ERR_OVERFLOW",
    5: "SPGEMM_ERR_TIMEOUT",
    6: "SPGEMM_ERR_CUDA",
    7: "SPGEMM_ERR_INTERNAL",
}

ABI_VERSION = 5  # SPGEMM_ABI_VERSION of include/spgemm.h

OPT_CHECKED = 1
OPT_MIN_SYM_BIN = 2
OPT_MIN_NUM_BIN = 3
OPT_CLUSTER_SIZE = 4
OPT_STREAMS = 5
OPT_PROFILE = 6
OPT_MIN_TRANSPOSE_BIN = 7
OPT_ONE_PASS = 8
OPT_ESC = 9


class CsrView(C.Structure):
    _fields_ = [
        ("m", C.c_int32),
        ("n", C.c_int32),
        ("nnz", C.c_int32),
        ("rpt", C.c_void_p),
        ("col", C.c_void_p),
        ("val", C.c_void_p),
    ]


class CsrOut(C.Structure):
    _fields_ = [
        ("m", C.c_int32),
        ("n", C.c_int32),
        ("nnz", C.c_int32),
        ("rpt", C.c_void_p),
        ("col", C.c_void_p),
        ("val", C.c_void_p),
    ]


class Info(C.Structure):
    _fields_ = [
        ("nip", C.c_int64),
        ("nnz", C.c_int64),
        ("max_row_nip", C.c_int32),
        ("max_row_nnz", C.c_int32),
        ("sym_bin_rows", C.c_int32 * 16),
        ("num_bin_rows", C.c_int32 * 16),
        ("sym_fail_rows", C.c_int32),
        ("n_sym_bins", C.c_int32),
        ("n_num_bins", C.c_int32),
        ("host_syncs", C.c_int32),
        ("phase_us", C.c_float * 8),
        ("one_pass", C.c_int32),
        ("esc_mask", C.c_int32),
    ]


PLAN_MAX_CANDIDATES = 16  # SPGEMM_PLAN_MAX_CANDIDATES


class PlanInfo(C.Structure):
    _fields_ = [
        ("candidates", C.c_int32),
        ("chosen", C.c_int32),
        ("team_scale", C.c_float * PLAN_MAX_CANDIDATES),
        ("cta_scale", C.c_float * PLAN_MAX_CANDIDATES),
        ("streams", C.c_int32 * PLAN_MAX_CANDIDATES),
        ("ms", C.c_float * PLAN_MAX_CANDIDATES),
    ]


class KernelTime(C.Structure):
    _fields_ = [
        ("name", C.c_char * 48),
        ("phase", C.c_int32),
        ("bin", C.c_int32),
        ("rows", C.c_int32),
        ("ms", C.c_float),
        ("start_ms", C.c_float),
    ]


class BatchDesc(C.Structure):
    _fields_ = [
        ("count", C.c_int32),
        ("a_row_off", C.c_void_p),
        ("b_row_off", C.c_void_p),
        ("c_col_off", C.c_void_p),
    ]


class BatchOut(C.Structure):
    _fields_ = [
        ("count", C.c_int32),
        ("products", C.POINTER(CsrOut)),
        ("n_blocks", C.c_int32),
        ("blocks", C.POINTER(C.c_void_p)),
        ("n_groups", C.c_int32),
    ]


# name -> (restype, argtypes); must list every function spgemm.h declares
SIGNATURES = {
    "spgemm_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "spgemm_destroy": (C.c_int, [C.c_void_p]),
    "spgemm_csr_f64": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                 C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_csr_f32": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                 C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_csr_free": (C.c_int, [C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_csr_host_f64": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                      C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_csr_host_f32": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                      C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_host_csr_free": (C.c_int, [C.POINTER(CsrOut)]),
    "spgemm_get_nip": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                 C.POINTER(C.c_int64), C.c_void_p]),
    "spgemm_get_nip_many": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(CsrView),
                                      C.POINTER(CsrView), C.POINTER(C.c_int64), C.c_void_p]),
    "spgemm_last_info": (C.c_int, [C.c_void_p, C.POINTER(Info)]),
    "spgemm_last_profile": (C.c_int, [C.c_void_p, C.POINTER(KernelTime), C.c_int32,
                                      C.POINTER(C.c_int32)]),
    "spgemm_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int64]),
    "spgemm_get_option": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
    "spgemm_ladder_info": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int64)]),
    "spgemm_batch_f64": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.POINTER(CsrView),
                                   C.POINTER(CsrView), C.POINTER(BatchOut), C.c_void_p]),
    "spgemm_batch_f32": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.POINTER(CsrView),
                                   C.POINTER(CsrView), C.POINTER(BatchOut), C.c_void_p]),
    "spgemm_batch_free": (C.c_int, [C.POINTER(BatchOut), C.c_void_p]),
    "spgemm_transpose_f64": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrOut),
                                       C.c_void_p]),
    "spgemm_transpose_f32": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrOut),
                                       C.c_void_p]),
    "spgemm_rap_f64": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                 C.POINTER(CsrView), C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_rap_f32": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                 C.POINTER(CsrView), C.POINTER(CsrOut), C.c_void_p]),
    "spgemm_plan_csr_f64": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                      C.c_int32, C.POINTER(CsrOut), C.POINTER(C.c_void_p),
                                      C.c_void_p]),
    "spgemm_plan_csr_f32": (C.c_int, [C.c_void_p, C.POINTER(CsrView), C.POINTER(CsrView),
                                      C.c_int32, C.POINTER(CsrOut), C.POINTER(C.c_void_p),
                                      C.c_void_p]),
    "spgemm_plan_batch_f64": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.POINTER(CsrView),
                                        C.POINTER(CsrView), C.c_int32, C.POINTER(BatchOut),
                                        C.POINTER(C.c_void_p), C.c_void_p]),
    "spgemm_plan_batch_f32": (C.c_int, [C.c_void_p, C.POINTER(BatchDesc), C.POINTER(CsrView),
                                        C.POINTER(CsrView), C.c_int32, C.POINTER(BatchOut),
                                        C.POINTER(C.c_void_p), C.c_void_p]),
    "spgemm_plan_execute": (C.c_int, [C.c_void_p, C.c_void_p]),
    "spgemm_plan_check": (C.c_int, [C.c_void_p, C.c_void_p]),
    "spgemm_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    "spgemm_plan_destroy": (C.c_int, [C.c_void_p]),
    "spgemm_row_nnz_noalloc": (C.c_int, [C.POINTER(CsrView), C.POINTER(CsrView), C.c_void_p,
                                         C.c_void_p]),
    "spgemm_last_error_string": (C.c_char_p, []),
    "spgemm_status_string": (C.c_char_p, [C.c_int]),
    "spgemm_abi_version": (C.c_int, []),
}


class SpgemmError(RuntimeError):
    """Raised for a non-OK status; mirrors the reference's std::runtime_error
    (src/libutils/include/utils/errors.cuh:11-22)."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{self.status_name}: {message}")


def load(path: Path = LIB_PATH) -> C.CDLL:
    if not path.exists():
        raise ImportError(
            f"{path.name} is not built; run `python -m gpuspgemm_b200.build` "
            "(the package has no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.spgemm_abi_version() != ABI_VERSION:
        raise ImportError("libspgemm_b200.so ABI version mismatch")
    return lib


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def check(status: int) -> None:
    if status != SPGEMM_OK:
        msg = lib().spgemm_last_error_string().decode(errors="replace")
        raise SpgemmError(status, msg)
