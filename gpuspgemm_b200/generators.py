"""Seeded synthetic CSR inputs for the SpGEMM workloads.

The reference benchmarks 12 SuiteSparse matrices downloaded over the network
(``tasks.py:24-93``); none are available offline.  These generators stand in for
them with the shapes, sizes and value distributions of the workloads this
library is measured on:

* ``uniform_rows``   square n x n, exactly k distinct uniform columns per row,
                     values U[-1, 1]                       (C = A*A, n = 4096, k = 8)
* ``power_law``      n x n graph, row degree ~ Zipf(s) on [1, cap], columns by
                     preferential attachment, values U(0, 1]  (n = 1e6, s = 2.0)
* ``stencil27`` / ``aggregation_prolongator``   AMG Galerkin operands R*A*P
* ``batch_pairs``    thousands of small independent square pairs
* ``served_request`` the request mix of the served stream

Every generator is a pure function of its arguments and seed.  All matrices
have sorted, duplicate-free columns per row.
"""
from __future__ import annotations

import numpy as np

from .csr import HostCSR

DEFAULT_SEED = 20261203


def _from_row_keys(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals=None,
                   dtype=np.float64) -> HostCSR:
    """CSR from (row, col) pairs that are unique; sorts by (row, col)."""
    key = rows.astype(np.int64) * n + cols.astype(np.int64)
    order = np.argsort(key, kind="stable")
    rows = rows[order]
    cols = cols[order].astype(np.int32)
    rpt = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=rpt[1:])
    if vals is None:
        vals = np.zeros(cols.shape[0], dtype=dtype)
    else:
        vals = np.asarray(vals)[order].astype(dtype)
    return HostCSR(m, n, rpt.astype(np.int32), cols, vals)


def sample_distinct_per_row(rng: np.random.Generator, counts: np.ndarray, ncols: int):
    """For row i draw counts[i] distinct uniform columns in [0, ncols).

    Returns (rows, cols) sorted by (row, col).  counts[i] must be <= ncols.
    """
    counts = np.asarray(counts, dtype=np.int64)
    if np.any(counts > ncols):
        raise ValueError("a row asks for more distinct columns than exist")
    m = counts.shape[0]
    rows = np.repeat(np.arange(m, dtype=np.int64), counts)
    cols = rng.integers(0, ncols, size=rows.shape[0], dtype=np.int64)
    while True:
        key = np.unique(rows * ncols + cols)
        rows = key // ncols
        cols = key % ncols
        have = np.bincount(rows, minlength=m)
        short = counts - have
        if not np.any(short > 0):
            return rows, cols
        # dense rows: fill the rest from the complement directly
        add_rows = np.repeat(np.arange(m, dtype=np.int64), short)
        add_cols = rng.integers(0, ncols, size=add_rows.shape[0], dtype=np.int64)
        rows = np.concatenate([rows, add_rows])
        cols = np.concatenate([cols, add_cols])


def uniform_rows(n: int = 4096, k: int = 8, seed: int = DEFAULT_SEED, dtype=np.float64,
                 m: int | None = None, low: float = -1.0, high: float = 1.0) -> HostCSR:
    """m x n, exactly k distinct uniformly random columns per row, values U[low, high]."""
    rng = np.random.default_rng(seed)
    m = n if m is None else m
    rows, cols = sample_distinct_per_row(rng, np.full(m, k), n)
    vals = rng.uniform(low, high, size=rows.shape[0])
    return _from_row_keys(m, n, rows, cols, vals, dtype)


def zipf_degrees(rng: np.random.Generator, n: int, exponent: float, cap: int,
                 dmin: int = 1) -> np.ndarray:
    """n draws from the Zipf law P(d) ~ d^-s truncated to [dmin, cap]."""
    d = np.arange(dmin, cap + 1, dtype=np.float64)
    p = d ** (-exponent)
    cdf = np.cumsum(p / p.sum())
    idx = np.searchsorted(cdf, rng.random(n), side="right")
    return np.minimum(idx, cap - dmin).astype(np.int64) + dmin


def power_law(n: int = 1_000_000, exponent: float = 2.0, cap: int = 4700,
              seed: int = DEFAULT_SEED, dtype=np.float64, block: int = 2000) -> HostCSR:
    """Power-law graph matrix.

    Row degrees ~ Zipf(exponent) on [1, cap].  Columns by preferential
    attachment: a target is drawn with probability proportional to
    (1 + its in-degree so far), sampled as a uniform pick from the multiset
    {every node once} + {every target drawn before}; rows are processed in
    blocks of ``block`` rows that share the in-degree snapshot of the block's
    start.  Duplicate columns within a row are dropped (so nnz is a little below
    the sum of degrees), columns sorted.  Values U(0, 1].
    """
    rng = np.random.default_rng(seed)
    cap = min(cap, n)
    deg = zipf_degrees(rng, n, exponent, cap)
    total = int(deg.sum())
    past = np.empty(total, dtype=np.int64)
    npast = 0
    for s in range(0, n, block):
        e = min(n, s + block)
        k = int(deg[s:e].sum())
        idx = rng.integers(0, n + npast, size=k, dtype=np.int64)
        old = idx >= n
        idx[old] = past[idx[old] - n]
        past[npast:npast + k] = idx
        npast += k
    rows = np.repeat(np.arange(n, dtype=np.int64), deg)
    key = np.unique(rows * n + past)
    rows = key // n
    cols = key % n
    vals = 1.0 - rng.random(rows.shape[0])
    rpt = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rpt[1:])
    return HostCSR(n, n, rpt.astype(np.int32), cols.astype(np.int32), vals.astype(dtype))


def stencil27(nx: int, ny: int | None = None, nz: int | None = None, dtype=np.float64,
              diag: float = 26.0, off: float = -1.0) -> HostCSR:
    """27-point stencil on an nx x ny x nz grid (natural ordering, x fastest)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    nrow = nx * ny * nz
    idx = np.arange(nrow, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    rows_l, cols_l, vals_l = [], [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                xx, yy, zz = x + dx, y + dy, z + dz
                ok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny) & (zz >= 0) & (zz < nz)
                r = idx[ok]
                c = (zz[ok] * ny + yy[ok]) * nx + xx[ok]
                rows_l.append(r)
                cols_l.append(c)
                v = diag if (dx, dy, dz) == (0, 0, 0) else off
                vals_l.append(np.full(r.shape[0], v))
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    vals = np.concatenate(vals_l)
    return _from_row_keys(nrow, nrow, rows, cols, vals, dtype)


def aggregation_prolongator(nx: int, ny: int | None = None, nz: int | None = None,
                            agg: int = 3, max_nnz: int = 8, seed: int = DEFAULT_SEED,
                            dtype=np.float64) -> HostCSR:
    """Piecewise-constant aggregation from agg^3 blocks plus smoothed fill.

    Fine point (x, y, z) belongs to aggregate (x // agg, y // agg, z // agg);
    the last partial layer in each dimension is merged into its neighbour
    (nx // agg aggregates per dimension).  Each row holds its own aggregate and
    up to ``max_nnz - 1`` neighbouring aggregates (those reached by a +-1 step
    of the point in x, y or z), weights U[0.1, 1].
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    rng = np.random.default_rng(seed)
    ax, ay, az = max(nx // agg, 1), max(ny // agg, 1), max(nz // agg, 1)
    nrow = nx * ny * nz
    idx = np.arange(nrow, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)

    def agg_of(xx, yy, zz):
        return (np.minimum(zz // agg, az - 1) * ay + np.minimum(yy // agg, ay - 1)) * ax + \
            np.minimum(xx // agg, ax - 1)

    rows_l, cols_l = [idx], [agg_of(x, y, z)]
    for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
              (1, 1, 0)):
        xx, yy, zz = x + d[0], y + d[1], z + d[2]
        ok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny) & (zz >= 0) & (zz < nz)
        rows_l.append(idx[ok])
        cols_l.append(agg_of(xx[ok], yy[ok], zz[ok]))
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    key = np.unique(rows * (ax * ay * az) + cols)
    rows = key // (ax * ay * az)
    cols = key % (ax * ay * az)
    # keep at most max_nnz per row (own aggregate always kept: it sorts anywhere,
    # so cap by taking the first max_nnz of each row)
    rpt = np.zeros(nrow + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=nrow), out=rpt[1:])
    pos = np.arange(rows.shape[0]) - rpt[rows]
    keep = pos < max_nnz
    rows, cols = rows[keep], cols[keep]
    vals = rng.uniform(0.1, 1.0, size=rows.shape[0])
    return _from_row_keys(nrow, ax * ay * az, rows, cols, vals, dtype)


def transpose(a: HostCSR) -> HostCSR:
    """CSR transpose (columns of the result sorted)."""
    rows = np.repeat(np.arange(a.m, dtype=np.int64), np.diff(a.rpt))
    return _from_row_keys(a.n, a.m, a.col.astype(np.int64), rows, a.val, a.val.dtype)


def batch_pairs(count: int = 4096, seed: int = DEFAULT_SEED, dtype=np.float32,
                rows_lo: int = 64, rows_hi: int = 16384, lam_lo: float = 6.0,
                lam_hi: float = 40.0):
    """Independent square pairs (A_i, B_i): rows log-uniform in [rows_lo, rows_hi],
    nnz per row ~ Poisson(lambda_i), lambda_i ~ U[lam_lo, lam_hi], uniform distinct
    columns, values U[-1, 1].  Yields HostCSR pairs lazily."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi), size=count)).astype(np.int64)
    lams = rng.uniform(lam_lo, lam_hi, size=count)
    seeds = rng.integers(0, 2**62, size=(count, 2))
    for i in range(count):
        yield tuple(_poisson_square(int(sizes[i]), float(lams[i]), int(seeds[i, j]), dtype)
                    for j in range(2))


def _poisson_square(n: int, lam: float, seed: int, dtype) -> HostCSR:
    rng = np.random.default_rng(seed)
    counts = np.minimum(rng.poisson(lam, size=n), n)
    rows, cols = sample_distinct_per_row(rng, counts, n)
    vals = rng.uniform(-1.0, 1.0, size=rows.shape[0])
    return _from_row_keys(n, n, rows, cols, vals, dtype)


def batch_packed_gpu(count: int = 4096, seed: int = DEFAULT_SEED, dtype=None, device="cuda",
                     rows_lo: int = 64, rows_hi: int = 16384, lam_lo: float = 6.0,
                     lam_hi: float = 40.0):
    """The batched workload generated directly on the GPU in packed form.

    `count` independent square pairs (A_i, B_i): rows log-uniform in
    [rows_lo, rows_hi], nnz per row ~ Poisson(lambda_i) with lambda_i ~
    U[lam_lo, lam_hi] (capped at the row count), uniform random columns with
    duplicates within a row dropped, values U[-1, 1].  Returns
    (a_row_off, b_row_off, c_col_off, A_packed, B_packed) with block-diagonal
    operands in global column indices (gpuspgemm_b200.api.PackedBatch fields).
    Seeded: sizes and rates from numpy, entries from a seeded torch generator on
    the device.
    """
    import torch
    dtype = dtype or torch.float32
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi), size=count)).astype(np.int64)
    lams = rng.uniform(lam_lo, lam_hi, size=count)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    if off[-1] >= 2**31:
        raise ValueError("batch has too many rows for int32 indices")
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed) & 0x7FFFFFFF)
    dev = torch.device(device)
    prod_of_row = torch.repeat_interleave(torch.arange(count, device=dev),
                                          torch.as_tensor(sizes, device=dev))
    m_of_row = torch.as_tensor(sizes, device=dev)[prod_of_row]
    off_of_row = torch.as_tensor(off[:-1], device=dev)[prod_of_row]

    def one():
        lam = torch.as_tensor(lams, device=dev, dtype=torch.float32)[prod_of_row]
        cnt = torch.minimum(torch.poisson(lam, generator=gen).to(torch.int64), m_of_row)
        rows = torch.repeat_interleave(torch.arange(int(off[-1]), device=dev), cnt)
        u = torch.rand(rows.shape[0], device=dev, generator=gen, dtype=torch.float64)
        col = (u * m_of_row[rows].to(torch.float64)).to(torch.int64)
        key = rows * 16384 + col
        key = torch.unique(key)  # sorted, duplicates dropped
        rows = key // 16384
        col = key % 16384
        rpt = torch.zeros(int(off[-1]) + 1, dtype=torch.int64, device=dev)
        rpt[1:] = torch.cumsum(torch.bincount(rows, minlength=int(off[-1])), 0)
        gcol = col + off_of_row[rows]
        val = (torch.rand(key.shape[0], device=dev, generator=gen, dtype=torch.float64) * 2 - 1)
        return rpt.to(torch.int32), gcol.to(torch.int32), val.to(dtype)

    from .api import DeviceCSR
    ar, ac, av = one()
    br, bc, bv = one()
    n = int(off[-1])
    offs = off.astype(np.int32)
    return offs, offs.copy(), offs.copy(), DeviceCSR(n, n, ar, ac, av), DeviceCSR(n, n, br, bc, bv)
