"""Real-matrix ingest: Matrix Market (.mtx) and SuiteSparse MATLAB (.mat) files
to the reference's ``.csr`` format, offline.

The reference fetches SuiteSparse ``.mat`` files and converts them in
``tasks.py:57-72``: ``Problem.A`` to CSR, then ``int32 nnz, m, n``,
``indptr``, ``indices`` and the values.  Here the same conversion runs on
files the user already has, and Matrix Market files are read too:

* coordinate format; fields real, integer or pattern (pattern -> 1.0);
  symmetry general, symmetric, skew-symmetric or hermitian (real data only);
  complex matrices are rejected;
* symmetric and hermitian entries off the diagonal are mirrored, skew ones
  mirrored with the sign flipped;
* duplicate coordinates are summed and every row's columns sorted -- the
  canonical CSR that ``scipy.sparse`` ``tocsr`` gives; entries stored as
  explicit zeros are kept (they are structure);
* values are written as float64, the ``.csr`` file's only value type.

CLI::

    python -m gpuspgemm_b200.convert INPUT.{mtx,mat} OUTPUT.csr
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

from .csr import HostCSR, save_csr


def _canonical(m: int, n: int, rows: np.ndarray, cols: np.ndarray,
               vals: np.ndarray) -> HostCSR:
    """CSR with duplicates summed and columns sorted (explicit zeros kept)."""
    if m > np.iinfo(np.int32).max or n > np.iinfo(np.int32).max:
        raise ValueError("matrix dimensions exceed int32")
    if rows.size and (rows.min() < 0 or rows.max() >= m or cols.min() < 0 or cols.max() >= n):
        raise ValueError("entry outside the declared matrix size")
    key = rows.astype(np.int64) * n + cols.astype(np.int64)
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order].astype(np.float64)
    first = np.ones(key.size, dtype=bool)
    first[1:] = key[1:] != key[:-1]
    starts = np.flatnonzero(first)
    summed = np.add.reduceat(vals, starts) if key.size else vals
    ukey = key[starts]
    if ukey.size > np.iinfo(np.int32).max:
        raise ValueError("nnz exceeds int32")
    r = (ukey // n).astype(np.int64)
    rpt = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=m), out=rpt[1:])
    return HostCSR(m, n, rpt.astype(np.int32), (ukey % n).astype(np.int32), summed)


def read_mtx(path: str | os.PathLike) -> HostCSR:
    """Read a Matrix Market coordinate file into canonical CSR (float64)."""
    with open(path, "rb") as f:
        header = f.readline().decode("ascii", "replace").strip().split()
        if len(header) != 5 or header[0].lower() != "%%matrixmarket" or \
                header[1].lower() != "matrix":
            raise ValueError(f"{path}: not a Matrix Market matrix header")
        fmt, field, symmetry = (h.lower() for h in header[2:])
        if fmt != "coordinate":
            raise ValueError(f"{path}: only the coordinate format is supported (got {fmt})")
        if field not in ("real", "integer", "pattern", "double"):
            raise ValueError(f"{path}: field '{field}' is not supported (complex data?)")
        if symmetry not in ("general", "symmetric", "skew-symmetric", "hermitian"):
            raise ValueError(f"{path}: symmetry '{symmetry}' is not supported")
        line = f.readline()
        while line and line.lstrip().startswith(b"%") or line.strip() == b"":
            if not line:
                raise ValueError(f"{path}: missing size line")
            line = f.readline()
        m, n, nnz = (int(x) for x in line.split())
        body = f.read()
    ncol = 2 if field == "pattern" else 3
    # comment lines may appear between entries; drop them before parsing
    if b"%" in body:
        body = b"\n".join(ln for ln in body.splitlines() if not ln.lstrip().startswith(b"%"))
    data = np.array(body.split(), dtype=np.float64) if body.strip() else np.zeros(0)
    if data.size != nnz * ncol:
        raise ValueError(f"{path}: expected {nnz} entries of {ncol} fields, "
                         f"found {data.size} numbers")
    data = data.reshape(nnz, ncol)
    rows = data[:, 0].astype(np.int64) - 1
    cols = data[:, 1].astype(np.int64) - 1
    vals = np.ones(nnz) if field == "pattern" else data[:, 2].copy()
    if symmetry != "general":
        off = rows != cols
        sign = -1.0 if symmetry == "skew-symmetric" else 1.0
        rows, cols, vals = (np.concatenate([rows, cols[off]]), np.concatenate([cols, rows[off]]),
                            np.concatenate([vals, sign * vals[off]]))
    return _canonical(m, n, rows, cols, vals)


def read_mat(path: str | os.PathLike) -> HostCSR:
    """Read a SuiteSparse MATLAB file's Problem.A the way the reference's
    download task does (tasks.py:57-63).  That task also adds Problem.Zeros
    (the explicit zeros of the original problem) with a sparse ``+=``, but a
    sparse sum drops entries whose result is 0, so the file it writes holds
    Problem.A's structure only; this reader gives the same matrix."""
    import scipy.io

    mat = scipy.io.loadmat(path)
    a = mat["Problem"]["A"][0][0].tocoo()
    if np.iscomplexobj(a.data):
        raise ValueError(f"{path}: complex matrices are not supported")
    keep = a.data != 0
    return _canonical(a.shape[0], a.shape[1], a.row[keep], a.col[keep],
                      np.asarray(a.data[keep], dtype=np.float64))


def convert(src: str | os.PathLike, dst: str | os.PathLike) -> HostCSR:
    ext = os.path.splitext(str(src))[1].lower()
    if ext == ".mtx":
        a = read_mtx(src)
    elif ext == ".mat":
        a = read_mat(src)
    else:
        raise ValueError(f"{src}: unknown extension (expected .mtx or .mat)")
    save_csr(dst, a)
    return a


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("input")
    ap.add_argument("output")
    args = ap.parse_args(argv)
    a = convert(args.input, args.output)
    print(f"{args.input} -> {args.output}: {a.m} x {a.n}, nnz {a.nnz}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
