"""CSR containers and the reference's ``.csr`` binary format.

``.csr`` layout (reference ``src/libutils/include/utils/csr.cuh:119-191`` and
the writer in ``tasks.py:66-72``), little-endian, no padding::

    int32 nnz, int32 m, int32 n
    int32 rpt[m + 1]
    int32 col[nnz]
    float64 val[nnz]          # always float64 on disk, also for float data

A file whose size is not exactly that is rejected ("too small" / "too large",
csr.cuh:126-128, 155-156).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

_HEADER = np.dtype("<i4")


@dataclass
class HostCSR:
    """Host CSR matrix (numpy arrays); mirrors ``utils::HostCSR<T>`` (csr.cuh:22-63)."""

    m: int
    n: int
    rpt: np.ndarray  # int32 [m + 1]
    col: np.ndarray  # int32 [nnz]
    val: np.ndarray  # float32 or float64 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    @property
    def dtype(self) -> np.dtype:
        return self.val.dtype

    def astype(self, dtype) -> "HostCSR":
        return HostCSR(self.m, self.n, self.rpt, self.col, self.val.astype(dtype))

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.rpt)

    def validate(self) -> None:
        """Raise ValueError unless the matrix satisfies the library's preconditions."""
        if self.rpt.shape != (self.m + 1,):
            raise ValueError("rpt must have m + 1 entries")
        if self.rpt[0] != 0 or self.rpt[-1] != self.nnz:
            raise ValueError("rpt must start at 0 and end at nnz")
        if np.any(np.diff(self.rpt) < 0):
            raise ValueError("rpt must be non-decreasing")
        if self.nnz and (self.col.min() < 0 or self.col.max() >= self.n):
            raise ValueError("column index out of range")
        if self.nnz > 1:
            d = np.diff(self.col.astype(np.int64))
            starts = self.rpt[1:-1]
            same_row = np.ones(self.nnz - 1, dtype=bool)
            same_row[starts[(starts > 0) & (starts < self.nnz)] - 1] = False
            if np.any(d[same_row] <= 0):
                raise ValueError("columns must be sorted and duplicate-free within rows")


def load_csr(path: str | os.PathLike, dtype=np.float64) -> HostCSR:
    """Read a ``.csr`` file (csr.cuh:119-160); values converted to ``dtype``."""
    size = os.path.getsize(path)
    if size < 12:
        raise ValueError(f"File {path} is too small")
    with open(path, "rb") as f:
        nnz, m, n = np.frombuffer(f.read(12), dtype=_HEADER)
        nnz, m, n = int(nnz), int(m), int(n)
        expect = 12 + 4 * (m + 1) + 4 * nnz + 8 * nnz
        if size < expect:
            raise ValueError(f"Failed to read file {path}")
        if size > expect:
            raise ValueError(f"File {path} is too large")
        rpt = np.frombuffer(f.read(4 * (m + 1)), dtype="<i4").astype(np.int32)
        col = np.frombuffer(f.read(4 * nnz), dtype="<i4").astype(np.int32)
        val = np.frombuffer(f.read(8 * nnz), dtype="<f8").astype(dtype)
    return HostCSR(m, n, rpt, col, val)


def save_csr(path: str | os.PathLike, a: HostCSR) -> None:
    """Write a ``.csr`` file (csr.cuh:162-191); values always as float64."""
    with open(path, "wb") as f:
        np.array([a.nnz, a.m, a.n], dtype="<i4").tofile(f)
        np.asarray(a.rpt, dtype="<i4").tofile(f)
        np.asarray(a.col, dtype="<i4").tofile(f)
        np.asarray(a.val, dtype="<f8").tofile(f)


def reference_equal(lhs: HostCSR, rhs: HostCSR) -> bool:
    """The reference's ``operator==`` (csr.cuh:218-239): identical structure,
    values equal or ``|l - r| <= 1e-8 + 1e-5 * max(|l|, |r|)``."""
    if (lhs.nnz, lhs.m, lhs.n) != (rhs.nnz, rhs.m, rhs.n):
        return False
    if not np.array_equal(lhs.rpt, rhs.rpt) or not np.array_equal(lhs.col, rhs.col):
        return False
    l = lhs.val.astype(np.float64)
    r = rhs.val.astype(np.float64)
    ok = (l == r) | (np.abs(l - r) <= 1e-8 + 1e-5 * np.maximum(np.abs(l), np.abs(r)))
    return bool(np.all(ok))
