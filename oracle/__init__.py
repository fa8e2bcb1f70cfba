"""TEST INFRASTRUCTURE ONLY: the CPU oracle and the reference's own GPU build.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
``--impl reference`` legs use this package, and only as the checker or the
reported baseline -- never as the product path.

* ``spgemm(A, B)``       row-wise Gustavson in C (oracle/gustavson.c), FP64 or
                         FP32 accumulate, sorted columns, products summed in
                         A-row order; restates the reference's method results
                         (see the header of gustavson.c for file:line anchors)
* ``ref_proposal(A, B)`` the reference's own proposal_inner<T, Parameters<CC80>>
                         compiled for sm_100a into oracle/_ref (needs a GPU)
* ``ref_cusparse2(A, B)`` the reference's cuSPARSE ALG2 validate path (GPU)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_proposal.so"
# root of the reference checkout (read-only), from the environment when set
REF_ROOT = Path(os.environ.get("GPUSPGEMM_REFERENCE", "/root/reference"))
REF_SRC = REF_ROOT / "src"

sys.path.insert(0, str(HERE.parent))
from gpuspgemm_b200.csr import HostCSR  # noqa: E402

_P = C.c_void_p


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if ref is None:
        ref = REF_SRC.exists()
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "opsparse",
                        f"PYTHON={sys.executable}", f"REF_SRC={REF_SRC}"], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build(ref=False)
        l = C.CDLL(str(LIB))
        l.oracle_nip.restype = C.c_int64
        l.oracle_nip.argtypes = [C.c_int32, _P, _P, _P, _P]
        l.oracle_symbolic.restype = C.c_int
        l.oracle_symbolic.argtypes = [C.c_int32, C.c_int32, _P, _P, _P, _P, _P]
        for name in ("oracle_numeric_f64", "oracle_numeric_f32", "oracle_abs_bound_f64"):
            fn = getattr(l, name)
            fn.restype = C.c_int
            fn.argtypes = [C.c_int32, C.c_int32] + [_P] * 9
        l.oracle_set_threads.argtypes = [C.c_int]
        l.oracle_max_threads.restype = C.c_int
        l.oracle_count_reference_mismatch_f64.restype = C.c_int64
        l.oracle_count_reference_mismatch_f64.argtypes = [C.c_int64, _P, _P]
        _lib = l
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P) if a.size else None


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def nip(A: HostCSR, B: HostCSR, per_row: bool = False):
    """Total (and optionally per-row) intermediate products."""
    rows = np.zeros(A.m, dtype=np.int64) if per_row else None
    t = lib().oracle_nip(A.m, _p(A.rpt), _p(A.col), _p(B.rpt),
                         _p(rows) if per_row else None)
    return (int(t), rows) if per_row else int(t)


def symbolic(A: HostCSR, B: HostCSR) -> np.ndarray:
    rpt = np.zeros(A.m + 1, dtype=np.int32)
    st = lib().oracle_symbolic(A.m, B.n, _p(A.rpt), _p(A.col), _p(B.rpt), _p(B.col), _p(rpt))
    if st == 2:
        raise OverflowError("nnz(C) exceeds int32")
    if st != 0:
        raise MemoryError("oracle allocation failed")
    return rpt


def spgemm(A: HostCSR, B: HostCSR, dtype=None) -> HostCSR:
    """C = A * B on the CPU.  dtype float64 accumulates in FP64, float32 in FP32."""
    if A.n != B.m:
        raise ValueError("A.n must equal B.m")
    dtype = np.dtype(dtype or A.val.dtype)
    a_val = np.ascontiguousarray(A.val, dtype=dtype)
    b_val = np.ascontiguousarray(B.val, dtype=dtype)
    rpt = symbolic(A, B)
    nnz = int(rpt[-1])
    col = np.zeros(nnz, dtype=np.int32)
    val = np.zeros(nnz, dtype=dtype)
    fn = lib().oracle_numeric_f64 if dtype == np.float64 else lib().oracle_numeric_f32
    st = fn(A.m, B.n, _p(A.rpt), _p(A.col), _p(a_val), _p(B.rpt), _p(B.col), _p(b_val),
            _p(rpt), _p(col), _p(val))
    if st != 0:
        raise MemoryError("oracle allocation failed")
    return HostCSR(A.m, B.n, rpt, col, val)


def transpose(A: HostCSR) -> HostCSR:
    """A^T with sorted columns: a stable counting sort of A's entries by
    column (entries of one column keep A's row order).  The reference has no
    transpose; R = P^T of its Galerkin use is formed by the caller."""
    rows = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rpt))
    order = np.argsort(A.col, kind="stable")
    rpt = np.zeros(A.n + 1, dtype=np.int32)
    np.cumsum(np.bincount(A.col, minlength=A.n), out=rpt[1:])
    return HostCSR(A.n, A.m, rpt, rows[order].astype(np.int32), A.val[order])


def abs_bound(A: HostCSR, B: HostCSR, Cref: HostCSR) -> np.ndarray:
    """Per-entry sum_k |a_ik| |b_kj| over C's structure (FP64)."""
    a_val = np.ascontiguousarray(A.val, dtype=np.float64)
    b_val = np.ascontiguousarray(B.val, dtype=np.float64)
    out = np.zeros(Cref.nnz, dtype=np.float64)
    st = lib().oracle_abs_bound_f64(A.m, B.n, _p(A.rpt), _p(A.col), _p(a_val), _p(B.rpt),
                                    _p(B.col), _p(b_val), _p(Cref.rpt), _p(Cref.col), _p(out))
    if st != 0:
        raise MemoryError("oracle allocation failed")
    return out


def compare(Cgpu: HostCSR, Cref: HostCSR, bound: np.ndarray | None = None) -> dict:
    """Structure equality plus the error figures every parity test states:
    max relative error over entries with c_ref != 0, the condition-aware error
    max |dc| / sum_k |a_ik||b_kj|, and the reference tolerance's mismatch count."""
    res = {
        "m_equal": Cgpu.m == Cref.m and Cgpu.n == Cref.n,
        "rpt_equal": bool(np.array_equal(Cgpu.rpt, Cref.rpt)),
        "col_equal": bool(Cgpu.nnz == Cref.nnz and np.array_equal(Cgpu.col, Cref.col)),
        "nnz": int(Cref.nnz),
    }
    if not res["col_equal"]:
        res.update(max_rel=float("inf"), max_cond=float("inf"), ref_mismatch=-1,
                   bit_exact=False)
        return res
    g = Cgpu.val.astype(np.float64)
    r = Cref.val.astype(np.float64)
    d = np.abs(g - r)
    nz = r != 0
    res["max_rel"] = float((d[nz] / np.abs(r[nz])).max()) if np.any(nz) else 0.0
    res["max_abs"] = float(d.max()) if d.size else 0.0
    if bound is not None:
        bz = bound > 0
        res["max_cond"] = float((d[bz] / bound[bz]).max()) if np.any(bz) else 0.0
    res["ref_mismatch"] = int(lib().oracle_count_reference_mismatch_f64(
        int(r.size), _p(np.ascontiguousarray(g)), _p(np.ascontiguousarray(r))))
    res["bit_exact"] = bool(np.array_equal(Cgpu.val, Cref.val.astype(Cgpu.val.dtype)))
    return res


# ---- the reference's own GPU build (oracle/_ref) ---------------------------

_ref = None


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        l = C.CDLL(str(REF_LIB))
        args = [C.c_int32, C.c_int32, C.c_int32, _P, _P, _P] * 2
        for name in ("ref_proposal_f64", "ref_proposal_f32", "ref_cusparse2_f64",
                     "ref_cusparse2_f32"):
            fn = getattr(l, name)
            fn.restype = C.c_int
            fn.argtypes = args + [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
        for name in ("ref_time_f64", "ref_time_f32"):
            fn = getattr(l, name)
            fn.restype = C.c_int
            fn.argtypes = [C.c_int] + args + [C.c_int, C.c_int, _P, _P]
        l.ref_last_error.restype = C.c_char_p
        l.ref_free.argtypes = [_P]
        _ref = l
    return _ref


def _ref_args(A: HostCSR, B: HostCSR, dtype):
    keep = []
    out = []
    for M in (A, B):
        v = np.ascontiguousarray(M.val, dtype=dtype)
        keep.append(v)
        out += [M.m, M.n, M.nnz, _p(M.rpt), _p(M.col), _p(v)]
    return out, keep


def _ref_run(which: str, A: HostCSR, B: HostCSR, dtype) -> HostCSR:
    dtype = np.dtype(dtype or A.val.dtype)
    suffix = "f64" if dtype == np.float64 else "f32"
    fn = getattr(ref_lib(), f"ref_{which}_{suffix}")
    args, keep = _ref_args(A, B, dtype)
    dims = np.zeros(3, dtype=np.int32)
    prpt, pcol, pval = _P(), _P(), _P()
    st = fn(*args, _p(dims), C.byref(prpt), C.byref(pcol), C.byref(pval))
    if st != 0:
        raise RuntimeError(ref_lib().ref_last_error().decode())
    m, n, nnz = (int(x) for x in dims)
    ct = C.c_double if dtype == np.float64 else C.c_float
    rpt = np.ctypeslib.as_array(C.cast(prpt, C.POINTER(C.c_int32)), (m + 1,)).copy()
    col = np.ctypeslib.as_array(C.cast(pcol, C.POINTER(C.c_int32)), (max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(C.cast(pval, C.POINTER(ct)), (max(nnz, 1),))[:nnz].copy()
    for p in (prpt, pcol, pval):
        ref_lib().ref_free(p)
    del keep
    return HostCSR(m, n, rpt, col, val)


def ref_proposal(A: HostCSR, B: HostCSR, dtype=None) -> HostCSR:
    return _ref_run("proposal", A, B, dtype)


def ref_cusparse2(A: HostCSR, B: HostCSR, dtype=None) -> HostCSR:
    return _ref_run("cusparse2", A, B, dtype)


def ref_time(which: str, A: HostCSR, B: HostCSR, dtype=None, warmups: int = 3,
             runs: int = 5) -> tuple[list[float], int]:
    """Wall-clock seconds per call of the reference (its `measure` lambda) and NIP."""
    dtype = np.dtype(dtype or A.val.dtype)
    suffix = "f64" if dtype == np.float64 else "f32"
    fn = getattr(ref_lib(), f"ref_time_{suffix}")
    args, keep = _ref_args(A, B, dtype)
    secs = np.zeros(runs, dtype=np.float64)
    nipv = np.zeros(1, dtype=np.int64)
    st = fn(0 if which == "proposal" else 1, *args, warmups, runs, _p(secs), _p(nipv))
    if st != 0:
        raise RuntimeError(ref_lib().ref_last_error().decode())
    del keep
    return list(secs), int(nipv[0])


# ---- the reference's vendored OpSparse (oracle/_ref/libref_opsparse_*.so) ----

OPS_LIBS = {np.dtype(np.float64): HERE / "_ref" / "libref_opsparse_f64.so",
            np.dtype(np.float32): HERE / "_ref" / "libref_opsparse_f32.so"}
_ops = {}


def ops_available(dtype=np.float64) -> bool:
    return OPS_LIBS[np.dtype(dtype)].exists()


def ops_lib(dtype=np.float64) -> C.CDLL:
    dtype = np.dtype(dtype)
    if dtype not in _ops:
        path = OPS_LIBS[dtype]
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle opsparse)")
        l = C.CDLL(str(path))
        args = [C.c_int32, C.c_int32, C.c_int32, _P, _P, _P] * 2
        l.ops_run.restype = C.c_int
        l.ops_run.argtypes = args + [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
        l.ops_time.restype = C.c_int
        l.ops_time.argtypes = args + [C.c_int, C.c_int, _P]
        l.ops_last_error.restype = C.c_char_p
        l.ops_free.argtypes = [_P]
        assert l.ops_value_bytes() == dtype.itemsize
        _ops[dtype] = l
    return _ops[dtype]


def ops_run(A: HostCSR, B: HostCSR, dtype=np.float64) -> HostCSR:
    """C = A * B through the reference's vendored OpSparse (src/libopsparse)."""
    dtype = np.dtype(dtype)
    l = ops_lib(dtype)
    args, keep = _ref_args(A, B, dtype)
    dims = np.zeros(3, dtype=np.int32)
    prpt, pcol, pval = _P(), _P(), _P()
    if l.ops_run(*args, _p(dims), C.byref(prpt), C.byref(pcol), C.byref(pval)) != 0:
        raise RuntimeError(l.ops_last_error().decode())
    m, n, nnz = (int(x) for x in dims)
    ct = C.c_double if dtype == np.float64 else C.c_float
    rpt = np.ctypeslib.as_array(C.cast(prpt, C.POINTER(C.c_int32)), (m + 1,)).copy()
    col = np.ctypeslib.as_array(C.cast(pcol, C.POINTER(C.c_int32)), (max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(C.cast(pval, C.POINTER(ct)), (max(nnz, 1),))[:nnz].copy()
    for q in (prpt, pcol, pval):
        l.ops_free(q)
    del keep
    return HostCSR(m, n, rpt, col, val)


def ops_time(A: HostCSR, B: HostCSR, dtype=np.float64, warmups: int = 3,
             runs: int = 5) -> list[float]:
    """Wall-clock seconds per OpSparse call, as the reference's opsparse app
    measures them (src/apps/opsparse.cu:35-44)."""
    dtype = np.dtype(dtype)
    l = ops_lib(dtype)
    args, keep = _ref_args(A, B, dtype)
    secs = np.zeros(runs, dtype=np.float64)
    if l.ops_time(*args, warmups, runs, _p(secs)) != 0:
        raise RuntimeError(l.ops_last_error().decode())
    del keep
    return list(secs)
