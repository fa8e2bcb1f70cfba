"""GPU parity: the sm_100a library against the CPU oracle (and the reference's
own GPU build where it is present), through the C ABI.

Bar: row pointers and sorted column indices bit-exact; values within
    FP64: 1e-12 relative per entry,   FP32 (accumulated in FP32): 1e-5,
stated as (a) max |dc|/|c_ref| over entries with c_ref != 0 -- asserted where
the inputs cannot cancel (all values positive) -- and (b) the cancellation-
aware max |dc| / sum_k |a_ik||b_kj|, asserted everywhere.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

from gpuspgemm_b200 import generators as G
from gpuspgemm_b200.csr import HostCSR, load_csr

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = {np.dtype(np.float64): 1e-12, np.dtype(np.float32): 1e-5}
RESULTS = []


def gpu_product(A: HostCSR, B: HostCSR, handle, dtype) -> HostCSR:
    from gpuspgemm_b200.api import DeviceCSR, proposal
    dA = DeviceCSR.from_host(A.astype(dtype))
    dB = DeviceCSR.from_host(B.astype(dtype))
    return proposal(dA, dB, handle).to_host()


def check(oracle, A, B, C, dtype, name, positive=False):
    dtype = np.dtype(dtype)
    A64 = A.astype(dtype).astype(np.float64)  # the rounded inputs, exactly
    B64 = B.astype(dtype).astype(np.float64)
    R = oracle.spgemm(A64, B64, np.float64)
    res = oracle.compare(C, R, oracle.abs_bound(A64, B64, R))
    res["case"] = name
    res["dtype"] = dtype.name
    RESULTS.append(res)
    assert res["rpt_equal"], res
    assert res["col_equal"], res
    assert res.get("max_cond", 0.0) <= TOL[dtype], res
    if positive:
        assert res["max_rel"] <= TOL[dtype], res
    return res


@pytest.fixture(scope="module", autouse=True)
def _dump_results():
    yield
    # the per-case error figures, when SPGEMM_PARITY_OUT names a folder
    out = Path(os.environ.get("SPGEMM_PARITY_OUT", "")) if os.environ.get("SPGEMM_PARITY_OUT") else None
    if out is not None and out.is_dir():
        (out / "parity_results.json").write_text(json.dumps(RESULTS, indent=1, default=str))


def test_uniform_4096x8_f64(handle, oracle_mod):
    A = G.uniform_rows(4096, 8)
    C = gpu_product(A, A, handle, np.float64)
    check(oracle_mod, A, A, C, np.float64, "uniform4096x8")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_power_law_small(handle, oracle_mod, dtype):
    A = G.power_law(30000, 2.0, 3000, seed=21)
    C = gpu_product(A, A, handle, dtype)
    check(oracle_mod, A, A, C, dtype, "powerlaw30000", positive=True)


def test_power_law_1m_f64(handle, oracle_mod):
    """Full-size power-law C = A*A (n = 1e6, Zipf 2.0, cap 4700)."""
    A = G.power_law()
    C = gpu_product(A, A, handle, np.float64)
    check(oracle_mod, A, A, C, np.float64, "powerlaw1M", positive=True)


def test_rectangular(handle, oracle_mod):
    A = G.uniform_rows(700, 9, seed=31, m=500)
    B = G.uniform_rows(300, 7, seed=32, m=700)
    C = gpu_product(A, B, handle, np.float64)
    assert (C.m, C.n) == (500, 300)
    check(oracle_mod, A, B, C, np.float64, "rect500x700x300")


def _ladder_len(handle, which):
    return len(handle.ladder(which, 8))


@pytest.mark.parametrize("b", range(9))
def test_forced_sym_bin(handle, oracle_mod, b):
    """Every row routed to at least count bin b: each kernel variant runs."""
    from gpuspgemm_b200 import _native as N
    if b >= _ladder_len(handle, 0):
        pytest.skip("no such bin")
    A = G.power_law(3000, 2.0, 300, seed=41)
    handle.set_option(N.OPT_MIN_SYM_BIN, b)
    handle.set_option(N.OPT_ONE_PASS, 2)  # the count kernels run in two-pass mode only
    try:
        C = gpu_product(A, A, handle, np.float64)
        assert handle.info()["one_pass"] == 0
    finally:
        handle.set_option(N.OPT_MIN_SYM_BIN, -1)
        handle.set_option(N.OPT_ONE_PASS, 0)
    check(oracle_mod, A, A, C, np.float64, f"forced_sym_bin{b}", positive=True)


def _wide_pair():
    """B with more than 2^20 columns: the fill ladder with hash CTA bins."""
    A = G.power_law(3000, 2.0, 300, seed=43)
    B = G.uniform_rows((1 << 20) + 5, 8, seed=44, m=3000)
    return A, B


@pytest.mark.parametrize("b", range(9))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("width", ["narrow", "wide"])
@pytest.mark.parametrize("passes", [1, 2])
def test_forced_num_bin(handle, oracle_mod, b, dtype, width, passes):
    """Every row routed to at least fill bin b, with C's row sizes from the
    one-pass fill (bins keyed by NIP) or from the count kernels (by nnz)."""
    from gpuspgemm_b200 import _native as N
    which = 2 if width == "narrow" else 1
    if b >= len(handle.ladder(which, 8)):
        pytest.skip("no such bin")
    if width == "narrow":
        A = G.power_law(3000, 2.0, 300, seed=42)
        B = A
    else:
        A, B = _wide_pair()
    handle.set_option(N.OPT_MIN_NUM_BIN, b)
    handle.set_option(N.OPT_ONE_PASS, passes)
    try:
        C = gpu_product(A, B, handle, dtype)
        assert handle.info()["one_pass"] == (1 if passes == 1 else 0)
    finally:
        handle.set_option(N.OPT_MIN_NUM_BIN, -1)
        handle.set_option(N.OPT_ONE_PASS, 0)
    check(oracle_mod, A, B, C, dtype, f"forced_num_bin{b}_{width}_pass{passes}", positive=True)


@pytest.mark.parametrize("shuffle", [False, True])
def test_global_bins_block_diagonal(handle, oracle_mod, shuffle):
    """Every row in the global bitmap bins of both phases, on a block-diagonal
    product (each row's column window is one block).  With `shuffle`, rows of B
    are unsorted, so keys fall outside the first/last-column window and the
    kernels redo those rows over all of B's columns."""
    from gpuspgemm_b200 import _native as N
    blocks = [G.power_law(1500, 2.0, 300, seed=900 + i) for i in range(3)]
    A = _block_diag(blocks)
    B = HostCSR(A.m, A.n, A.rpt.copy(), A.col.copy(), A.val.copy())
    if shuffle:
        rng = np.random.default_rng(5)
        for r in range(0, B.m, 7):
            s, e = B.rpt[r], B.rpt[r + 1]
            p = rng.permutation(e - s)
            B.col[s:e] = B.col[s:e][p]
            B.val[s:e] = B.val[s:e][p]
    handle.set_option(N.OPT_MIN_SYM_BIN, _ladder_len(handle, 0) - 1)
    handle.set_option(N.OPT_MIN_NUM_BIN, _ladder_len(handle, 2) - 1)
    handle.set_option(N.OPT_ONE_PASS, 2)
    try:
        C = gpu_product(A, B, handle, np.float64)
        # the same rows in the one-pass fill's global bin
        handle.set_option(N.OPT_ONE_PASS, 1)
        C1 = gpu_product(A, B, handle, np.float64)
    finally:
        handle.set_option(N.OPT_MIN_SYM_BIN, -1)
        handle.set_option(N.OPT_MIN_NUM_BIN, -1)
        handle.set_option(N.OPT_ONE_PASS, 0)
    check(oracle_mod, A, A, C1, np.float64, f"global_blockdiag_onepass{int(shuffle)}",
          positive=True)
    check(oracle_mod, A, A, C, np.float64, f"global_blockdiag_shuffle{int(shuffle)}",
          positive=True)


def _block_diag(mats):
    rpt, cols, vals = [np.zeros(1, np.int32)], [], []
    nz = c0 = 0
    for M in mats:
        rpt.append(M.rpt[1:] + nz)
        cols.append(M.col + c0)
        vals.append(M.val)
        nz += M.nnz
        c0 += M.n
    return HostCSR(sum(M.m for M in mats), c0, np.concatenate(rpt).astype(np.int32),
                   np.concatenate(cols).astype(np.int32), np.concatenate(vals))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_long_rows_wide_cta_bins(handle, oracle_mod, dtype):
    """Rows of ~20.7k, ~12k and ~2.4k distinct columns of a B with 2^21 + 7
    columns: the hash CTA bins' register sort (up to 16 keys per thread) and
    its shared-memory fallback for longer rows."""
    rng = np.random.default_rng(11)
    nb, n = 2600, (1 << 21) + 7
    b_rows = [np.unique(rng.integers(0, n, 8)) for _ in range(nb)]
    B = HostCSR(nb, n, np.concatenate([[0], np.cumsum([len(r) for r in b_rows])]).astype(np.int32),
                np.concatenate(b_rows).astype(np.int32),
                rng.uniform(0.1, 1, sum(len(r) for r in b_rows)))
    cols = [np.arange(nb), np.sort(rng.choice(nb, 1500, replace=False)),
            np.sort(rng.choice(nb, 300, replace=False))]
    A = HostCSR(3, nb, np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.int32),
                np.concatenate(cols).astype(np.int32), rng.uniform(0.1, 1, sum(map(len, cols))))
    C = gpu_product(A, B, handle, dtype)
    assert int(np.diff(C.rpt).max()) > 16384
    check(oracle_mod, A, B, C, dtype, "long_rows_wide", positive=True)


@pytest.mark.parametrize("passes", [1, 2])
@pytest.mark.parametrize("ncols", [(1 << 21) + 7, 5_000_011, (1 << 23) + 3])
def test_heaviest_wide_rows_in_cluster_bitmaps(handle, oracle_mod, passes, ncols):
    """Rows of ~40k-200k distinct columns, past the largest CTA bin (32,768),
    over a B of 2^21 + 7, 5.0 M or 2^23 + 3 columns: the cluster bitmap bin
    holds each row's bitmap in the shared memory of a cluster of 3, 5 or 8 CTAs
    (columns split by 2^20 per CTA, reached through distributed shared
    memory).  A B of 9 M columns is past 8 CTAs: those rows run in the global
    bitmap bin (test_rows_past_the_cluster_bitmaps_run_global)."""
    from gpuspgemm_b200 import _native as N
    rng = np.random.default_rng(12)
    nb = 6000
    b_rows = [np.unique(rng.integers(0, ncols, 40)) for _ in range(nb)]
    B = HostCSR(nb, ncols,
                np.concatenate([[0], np.cumsum([len(r) for r in b_rows])]).astype(np.int32),
                np.concatenate(b_rows).astype(np.int32),
                rng.uniform(0.1, 1, sum(len(r) for r in b_rows)))
    cols = [np.arange(nb), np.sort(rng.choice(nb, 1100, replace=False)),
            np.sort(rng.choice(nb, 40, replace=False)), np.arange(0, nb, 3)]
    A = HostCSR(len(cols), nb,
                np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.int32),
                np.concatenate(cols).astype(np.int32), rng.uniform(0.1, 1, sum(map(len, cols))))
    handle.set_option(N.OPT_ONE_PASS, passes)
    try:
        C = gpu_product(A, B, handle, np.float64)
        info = handle.info()
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    assert int(np.diff(C.rpt).max()) > 200_000
    wide = handle.ladder(1, 8)
    assert info["num_bin_rows"][len(wide) - 2] == 3      # the three rows past 32,768
    check(oracle_mod, A, B, C, np.float64, f"wide_cluster_bitmap_{ncols}_pass{passes}",
          positive=True)


def test_rows_past_the_cluster_bitmaps_run_global(handle, oracle_mod):
    """B of 9 M columns (more than 8 CTAs x 2^20): the cluster bitmap bin hands
    its rows to the global bitmap bin."""
    rng = np.random.default_rng(13)
    nb, ncols = 3000, 9_000_001
    b_rows = [np.unique(rng.integers(0, ncols, 30)) for _ in range(nb)]
    B = HostCSR(nb, ncols,
                np.concatenate([[0], np.cumsum([len(r) for r in b_rows])]).astype(np.int32),
                np.concatenate(b_rows).astype(np.int32),
                rng.uniform(0.1, 1, sum(len(r) for r in b_rows)))
    A = HostCSR(2, nb, np.array([0, nb, nb + 5], np.int32),
                np.concatenate([np.arange(nb), np.arange(5)]).astype(np.int32),
                rng.uniform(0.1, 1, nb + 5))
    C = gpu_product(A, B, handle, np.float64)
    assert int(np.diff(C.rpt).max()) > 80_000
    check(oracle_mod, A, B, C, np.float64, "wide_past_cluster_bitmaps", positive=True)


@pytest.mark.parametrize("passes", [1, 2])
def test_high_compression_stencil(handle, oracle_mod, passes):
    """A 27-point stencil squared: ~5.9 products per entry of C, all
    accumulated with global reductions into the row's slice of C.val; in
    one-pass mode each row's slot holds its NIP entries, ~6x its nnz."""
    from gpuspgemm_b200 import _native as N
    S = G.stencil27(20)
    handle.set_option(N.OPT_ONE_PASS, passes)
    try:
        C = gpu_product(S, S, handle, np.float64)
        info = handle.info()
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    assert info["nip"] > 5 * info["nnz"] and info["one_pass"] == (passes == 1)
    check(oracle_mod, S, S, C, np.float64, f"stencil20_squared_pass{passes}")


@pytest.mark.parametrize("esc", [0, 1, 2])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_one_pass_esc_bins(handle, oracle_mod, esc, dtype):
    """One pass with B.n <= 2^20 and the team bins expanding, sorting and
    compressing where sampled compression is low (0), always (1) or never (2):
    power-law rows in every team bin, a stencil whose columns repeat up to 27
    times per row, and a stencil times a prolongator (NIP/nnz ~ 9)."""
    from gpuspgemm_b200 import _native as N
    cases = {"power_law": (G.power_law(3000, 2.0, 300, seed=42),) * 2,
             "stencil12": (G.stencil27(12),) * 2,
             "stencil_prolongator": (G.stencil27(12), G.aggregation_prolongator(12, seed=3))}
    handle.set_option(N.OPT_ONE_PASS, 1)
    handle.set_option(N.OPT_ESC, esc)
    try:
        for name, (A, B) in cases.items():
            C = gpu_product(A, B, handle, dtype)
            info = handle.info()
            assert info["one_pass"] == 1
            assert info["esc_mask"] == {1: 0b11111, 2: 0}.get(esc, info["esc_mask"])
            check(oracle_mod, A, B, C, dtype, f"esc{esc}_{name}")
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
        handle.set_option(N.OPT_ESC, 0)


def test_esc_chosen_by_sampled_compression(handle, oracle_mod):
    """By default a fill bin expands, sorts and compresses only when its
    sampled rows repeat few columns: every team bin and the 256-thread bin of
    a power-law square (NIP/nnz 1.0), none of a 27-point stencil's square
    (NIP/nnz 4.6-6.0)."""
    from gpuspgemm_b200 import _native as N
    handle.set_option(N.OPT_ONE_PASS, 1)
    try:
        P = G.power_law(30000, 2.0, 3000, seed=21)
        C = gpu_product(P, P, handle, np.float64)
        info = handle.info()
        assert info["esc_mask"] == 0b11111
        check(oracle_mod, P, P, C, np.float64, "esc_auto_power_law", positive=True)
        # with both expanding, the 32-lane / 256-thread split moved to 512
        # products (decided on the device): bin 3 holds rows of 193-512
        # products, bin 4 rows of 513-3,072
        nip = oracle_mod.nip(P, P, per_row=True)[1]
        assert info["num_bin_rows"][3] == int(((nip > 192) & (nip <= 512)).sum())
        assert info["num_bin_rows"][4] == int(((nip > 512) & (nip <= 3072)).sum())
        assert int(((nip > 512) & (nip <= 768)).sum()) > 0
        S = G.stencil27(12)
        C = gpu_product(S, S, handle, np.float64)
        assert handle.info()["esc_mask"] == 0
        check(oracle_mod, S, S, C, np.float64, "esc_auto_stencil")
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_esc_sums_in_oracle_order(handle, oracle_mod, dtype):
    """Rows of at most 3,072 products all expand, sort and compress (team
    bins and the 256-thread bin), which sums each entry of C over its products
    in the oracle's (Gustavson) order with the same roundings: the values are
    bit-exact, not just within tolerance."""
    from gpuspgemm_b200 import _native as N
    dtype = np.dtype(dtype)
    handle.set_option(N.OPT_ONE_PASS, 1)
    handle.set_option(N.OPT_ESC, 1)
    try:
        for A, B in [(G.stencil27(12), G.stencil27(12)),  # NIP up to 729 per row
                     (G.uniform_rows(4096, 8), G.uniform_rows(4096, 8)),
                     (G.power_law(3000, 2.0, 40, seed=7), G.power_law(3000, 2.0, 40, seed=7)),
                     (G.power_law(3000, 2.0, 300, seed=42), G.power_law(3000, 2.0, 300, seed=42))]:
            A, B = A.astype(dtype), B.astype(dtype)
            assert oracle_mod.nip(A, B, per_row=True)[1].max() <= 3072
            C = gpu_product(A, B, handle, dtype)
            R = oracle_mod.spgemm(A, B, dtype)
            assert np.array_equal(C.rpt, R.rpt) and np.array_equal(C.col, R.col)
            assert C.val.dtype == dtype and np.array_equal(C.val, R.val)
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
        handle.set_option(N.OPT_ESC, 0)


@pytest.mark.parametrize("passes", [1, 2])
def test_bitmap_bin_back_to_back(handle, oracle_mod, passes):
    """Every row through the bitmap bin, whose persistent CTAs clear only the
    bitmap words a row set before taking the next row: back-to-back products
    of different structures and value types all match the oracle."""
    from gpuspgemm_b200 import _native as N
    assert len(handle.ladder(2, 8)) == 7
    handle.set_option(N.OPT_MIN_NUM_BIN, 5)
    handle.set_option(N.OPT_ONE_PASS, passes)
    try:
        for seed, dtype in [(61, np.float64), (62, np.float64), (63, np.float32), (61, np.float64)]:
            A = G.power_law(4000, 2.0, 400, seed=seed)
            C = gpu_product(A, A, handle, dtype)
            check(oracle_mod, A, A, C, dtype, f"bitmap_back_to_back_{seed}_pass{passes}",
                  positive=True)
    finally:
        handle.set_option(N.OPT_MIN_NUM_BIN, -1)
        handle.set_option(N.OPT_ONE_PASS, 0)


def test_compressing_wide_rows_keep_two_passes(handle, oracle_mod):
    """By default a product whose NIP lies mostly in rows above the team
    bins (> 768 products) that repeat their columns many times -- R * (A * P)
    of a 27-point stencil on 50^3, NIP/nnz 33 -- keeps two passes: in one pass
    those rows would fill NIP-sized CTA tables, in two passes nnz-sized team
    tables.  Both modes give the same C."""
    from gpuspgemm_b200 import _native as N
    A = G.stencil27(50)
    P = G.aggregation_prolongator(50, seed=3)
    R = oracle_mod.transpose(P)
    AP = oracle_mod.spgemm(A, P)
    assert oracle_mod.nip(R, AP) >= 1 << 21 and R.nnz >= 1 << 16
    C2 = gpu_product(R, AP, handle, np.float64)
    assert handle.info()["one_pass"] == 0
    handle.set_option(N.OPT_ONE_PASS, 1)
    try:
        C1 = gpu_product(R, AP, handle, np.float64)
        assert handle.info()["one_pass"] == 1
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    assert np.array_equal(C1.rpt, C2.rpt) and np.array_equal(C1.col, C2.col)
    check(oracle_mod, R, AP, C2, np.float64, "rap50_two_pass")


def test_one_pass_chosen_and_equal_to_two_pass(handle, oracle_mod):
    """By default a product whose temporaries fit runs one pass; its C equals
    the two-pass C in structure, and both match the oracle."""
    from gpuspgemm_b200 import _native as N
    A = G.power_law(200000, 2.0, 3000, seed=25)  # NIP above the one-pass minimum
    C1 = gpu_product(A, A, handle, np.float64)
    info1 = handle.info()
    assert info1["one_pass"] == 1 and info1["nip"] >= 1 << 21
    S = G.uniform_rows(4096, 8)  # a small product keeps two passes
    gpu_product(S, S, handle, np.float64)
    assert handle.info()["one_pass"] == 0
    handle.set_option(N.OPT_ONE_PASS, 2)
    try:
        C2 = gpu_product(A, A, handle, np.float64)
        info2 = handle.info()
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    # one pass, binned for the fill before the first synchronisation, and C
    # given the NIP as capacity (the sample sees few repeated columns): NIP +
    # fill binning, final; two passes: NIP binning, scan, final
    assert info2["one_pass"] == 0 and info2["host_syncs"] == 3 and info1["host_syncs"] == 2
    assert np.array_equal(C1.rpt, C2.rpt) and np.array_equal(C1.col, C2.col)
    assert info1["nnz"] == info2["nnz"] and info1["max_row_nnz"] == info2["max_row_nnz"]
    check(oracle_mod, A, A, C1, np.float64, "one_pass_default", positive=True)


def test_one_pass_capacity_shrinks_to_nnz(handle, oracle_mod):
    """A one-pass product whose sampled (light) rows repeat no column gets the
    NIP as C's capacity before its nnz is known; here the heavy rows collapse
    onto ten columns, so nnz is far below the NIP and C is copied to arrays of
    its own size after the last synchronisation (one more): the result still
    equals the oracle's."""
    rng = np.random.default_rng(31)
    n = 1 << 20
    clones, distinct = 2000, 200000
    b_rows = [np.arange(10, dtype=np.int32)] * clones
    b_rows += [np.sort(rng.choice(n, 5, replace=False)).astype(np.int32) for _ in range(distinct)]
    b_rpt = np.concatenate([[0], np.cumsum([len(r) for r in b_rows])]).astype(np.int32)
    B = HostCSR(len(b_rows), n, b_rpt, np.concatenate(b_rows),
                rng.uniform(0.5, 1.0, int(b_rpt[-1])))
    light = [np.sort(clones + rng.choice(distinct, 2, replace=False)).astype(np.int32)
             for _ in range(200000)]
    heavy = [np.sort(rng.choice(clones, 150, replace=False)).astype(np.int32) for _ in range(3000)]
    a_rows = light + heavy
    a_rpt = np.concatenate([[0], np.cumsum([len(r) for r in a_rows])]).astype(np.int32)
    A = HostCSR(len(a_rows), B.m, a_rpt, np.concatenate(a_rows),
                rng.uniform(0.5, 1.0, int(a_rpt[-1])))
    C = gpu_product(A, B, handle, np.float64)
    info = handle.info()
    assert info["one_pass"] == 1 and info["nip"] > 2 * info["nnz"]
    assert info["host_syncs"] == 3  # NIP + fill binning, row counts, the copy to C's size
    check(oracle_mod, A, B, C, np.float64, "one_pass_capacity_shrink", positive=True)


def test_heavy_row_spills_to_global(handle, oracle_mod):
    """One row with ~190k distinct columns: past the cluster table, so the
    count spills to the global bitmap and the fill runs in the global bin."""
    rng = np.random.default_rng(51)
    B = G.uniform_rows(300_000, 300, seed=52, m=1000)
    a_col = np.arange(1000, dtype=np.int32)
    A = HostCSR(3, 1000, np.array([0, 1000, 1000, 1003], np.int32),
                np.concatenate([a_col, np.array([1, 5, 9], np.int32)]),
                rng.uniform(0.1, 1.0, 1003))
    from gpuspgemm_b200 import _native as N
    handle.set_option(N.OPT_ONE_PASS, 2)  # the cluster table and its spill
    try:
        C = gpu_product(A, B, handle, np.float64)
        info = handle.info()
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    check(oracle_mod, A, B, C, np.float64, "heavy_row_spill", positive=False)
    assert info["max_row_nnz"] > 150_000


def test_row_past_the_cluster_table_spills(handle, oracle_mod):
    """A row with more distinct columns (230,400) than the cluster count
    table's 4 x 55,296 slots: the insert loop's load test spills it to the
    global bitmap bin as soon as the table passes its limit, and the fill
    runs in the global bin of the wide ladder (B.n > 2^20).  Its A entries
    span five slices of 1,024, so each slice adds at most 46,080 keys."""
    n_a, per = 5 * 1024, 45
    b_col = np.arange(n_a * per, dtype=np.int32)       # B row j: columns j*45 .. j*45+44
    rng = np.random.default_rng(61)
    B = HostCSR(n_a, (1 << 21) + 7, np.arange(0, n_a * per + 1, per, dtype=np.int32), b_col,
                rng.uniform(0.1, 1.0, n_a * per))
    A = HostCSR(2, n_a, np.array([0, n_a, n_a + 3], np.int32),
                np.concatenate([np.arange(n_a, dtype=np.int32), np.array([2, 7, 11], np.int32)]),
                rng.uniform(0.1, 1.0, n_a + 3))
    from gpuspgemm_b200 import _native as N
    handle.set_option(N.OPT_ONE_PASS, 2)  # the count phase: cluster table, then its spill
    try:
        C = gpu_product(A, B, handle, np.float64)
        info = handle.info()
    finally:
        handle.set_option(N.OPT_ONE_PASS, 0)
    check(oracle_mod, A, B, C, np.float64, "row_past_cluster_table", positive=True)
    assert info["max_row_nnz"] == n_a * per
    assert info["sym_fail_rows"] >= 1


def test_edge_cases(handle, oracle_mod):
    # empty rows in A, empty rows in B, rows of A that hit only empty B rows
    A = HostCSR(6, 5, np.array([0, 0, 2, 2, 3, 5, 5], np.int32),
                np.array([0, 3, 4, 1, 2], np.int32), np.array([2.0, -1.0, 1.5, 1.0, 3.0]))
    B = HostCSR(5, 4, np.array([0, 2, 2, 2, 4, 5], np.int32),
                np.array([1, 3, 0, 1, 2], np.int32), np.array([1.0, 2.0, 4.0, -2.0, 0.5]))
    C = gpu_product(A, B, handle, np.float64)
    check(oracle_mod, A, B, C, np.float64, "empty_rows")
    # cancellation to an exact zero keeps the entry
    A = HostCSR(2, 2, np.array([0, 2, 2], np.int32), np.array([0, 1], np.int32),
                np.array([1.0, 1.0]))
    B = HostCSR(2, 1, np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32),
                np.array([1.0, -1.0]))
    C = gpu_product(A, B, handle, np.float64)
    assert C.nnz == 1 and C.val.tolist() == [0.0]


def test_empty_operands(handle):
    A = HostCSR(4, 3, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = G.uniform_rows(5, 2, seed=1, m=3)
    C = gpu_product(A, B, handle, np.float64)
    assert (C.m, C.n, C.nnz) == (4, 5) + (0,) and np.all(C.rpt == 0)
    Z = HostCSR(0, 3, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    C = gpu_product(Z, B, handle, np.float64)
    assert (C.m, C.nnz) == (0, 0)


def test_dimension_mismatch_raises(handle):
    from gpuspgemm_b200 import SpgemmError
    A = G.uniform_rows(10, 2, seed=1, m=5)
    B = G.uniform_rows(10, 2, seed=2, m=11)
    with pytest.raises(SpgemmError, match="INVALID_ARG"):
        gpu_product(A, B, handle, np.float64)


def test_mode_options_validated(handle):
    """The pass and expand-sort-compress modes take 0, 1 or 2 only; a bad
    value is rejected and the option keeps its value."""
    from gpuspgemm_b200 import SpgemmError
    from gpuspgemm_b200 import _native as N
    for opt in (N.OPT_ONE_PASS, N.OPT_ESC):
        for bad in (-1, 3):
            with pytest.raises(SpgemmError, match="INVALID_ARG"):
                handle.set_option(opt, bad)
        assert handle.get_option(opt) == 0


def test_checked_mode_rejects_unsorted(handle):
    from gpuspgemm_b200 import SpgemmError
    from gpuspgemm_b200 import _native as N
    A = G.uniform_rows(50, 4, seed=3)
    bad = HostCSR(A.m, A.n, A.rpt.copy(), A.col.copy(), A.val.copy())
    bad.col[0], bad.col[1] = bad.col[1], bad.col[0]
    handle.set_option(N.OPT_CHECKED, 1)
    try:
        with pytest.raises(SpgemmError, match="INVALID_ARG"):
            gpu_product(A, bad, handle, np.float64)
        C = gpu_product(A, A, handle, np.float64)  # valid input still works
        assert C.nnz > 0
    finally:
        handle.set_option(N.OPT_CHECKED, 0)


def test_host_entry_point_and_nip(handle, oracle_mod):
    from gpuspgemm_b200.api import DeviceCSR, get_nip, proposal_host
    A = G.power_law(5000, 2.0, 500, seed=61)
    C = proposal_host(A, A, handle)
    check(oracle_mod, A, A, C, np.float64, "host_entry", positive=True)
    dA = DeviceCSR.from_host(A)
    assert get_nip(dA, dA, handle) == oracle_mod.nip(A, A)
    assert handle.info()["nip"] == oracle_mod.nip(A, A)


def test_repeat_calls_same_structure(handle):
    A = G.power_law(20000, 2.0, 1000, seed=71)
    C1 = gpu_product(A, A, handle, np.float64)
    C2 = gpu_product(A, A, handle, np.float64)
    assert np.array_equal(C1.rpt, C2.rpt) and np.array_equal(C1.col, C2.col)
    assert np.allclose(C1.val, C2.val, rtol=1e-13, atol=0)


def _golden():
    man = GOLDEN / "manifest.json"
    return sorted(json.loads(man.read_text()).items()) if man.exists() else []


@pytest.mark.parametrize("name,entry", _golden() or [pytest.param(
    None, None, marks=pytest.mark.skip(reason="golden vectors not generated"))])
def test_against_reference_golden(handle, oracle_mod, name, entry):
    """The library against the reference's own outputs on the same inputs."""
    dt = np.dtype(entry["dtype"])
    A = load_csr(GOLDEN / f"{name}.A.csr", dt)
    B = load_csr(GOLDEN / f"{name}.B.csr", dt)
    C = gpu_product(A, B, handle, dt)
    R = load_csr(GOLDEN / f"{name}.C_proposal.csr", dt)
    assert np.array_equal(C.rpt, R.rpt) and np.array_equal(C.col, R.col)
    check(oracle_mod, A, B, C, dt, f"golden_{name}")
