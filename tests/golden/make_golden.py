"""Generate the golden vectors that pin the CPU oracle to the REFERENCE itself.

The reference ships no tests or golden vectors.  This script runs the
reference's own GPU code -- proposal::proposal_inner<T, Parameters<CC80>> and
its cuSPARSE-ALG2 validate path, compiled from the reference sources into
oracle/_ref by `make -C oracle ref` -- on small seeded inputs, and writes
inputs and outputs as reference-format .csr files plus manifest.json.

It needs a B200 (run it on the GPU machine):
    python tests/golden/make_golden.py OUTDIR
and the files are committed under tests/golden/.  tests/test_oracle.py then
checks the oracle against them on the CPU, and the GPU parity tests check the
library against the same files.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from gpuspgemm_b200 import generators as G  # noqa: E402
from gpuspgemm_b200.csr import HostCSR, save_csr  # noqa: E402


def _csr(m, n, rows, dtype=np.float64):
    """HostCSR from a list of {col: val} dicts."""
    rpt = [0]
    col, val = [], []
    for r in rows:
        for c in sorted(r):
            col.append(c)
            val.append(r[c])
        rpt.append(len(col))
    return HostCSR(m, n, np.array(rpt, np.int32), np.array(col, np.int32),
                   np.array(val, dtype))


def cases():
    """name -> (A, B, dtype)."""
    out = {}
    a = G.uniform_rows(512, 8, seed=11)
    out["uniform512_f64"] = (a, a, np.float64)
    p = G.power_law(3000, 2.0, 300, seed=12)
    out["powerlaw3000_f64"] = (p, p, np.float64)
    p32 = p.astype(np.float32)
    out["powerlaw3000_f32"] = (p32, p32, np.float32)
    ra = G.uniform_rows(500, 6, seed=13, m=300)
    rb = G.uniform_rows(200, 5, seed=14, m=500)
    out["rect300x500x200_f64"] = (ra, rb, np.float64)
    # an entry whose value cancels to zero stays in C
    ca = _csr(2, 2, [{0: 1.0, 1: 1.0}, {}])
    cb = _csr(2, 1, [{0: 1.0}, {0: -1.0}])
    out["cancel_2x2_f64"] = (ca, cb, np.float64)
    # empty rows in A, empty rows in B, a row of A hitting only empty B rows
    ea = _csr(6, 5, [{}, {0: 2.0, 3: -1.0}, {}, {4: 1.5}, {1: 1.0, 2: 3.0}, {}])
    eb = _csr(5, 4, [{1: 1.0, 3: 2.0}, {}, {}, {0: 4.0, 1: -2.0}, {2: 0.5}])
    out["empty_rows_f64"] = (ea, eb, np.float64)
    # one long row (many A entries) over uniform B rows: heavy bins
    rng = np.random.default_rng(15)
    rows = [dict(zip(rng.choice(2000, 700, replace=False).tolist(),
                     rng.uniform(-1, 1, 700).tolist()))]
    rows += [dict(zip(rng.choice(2000, 4, replace=False).tolist(),
                      rng.uniform(-1, 1, 4).tolist())) for _ in range(63)]
    ha = _csr(64, 2000, rows)
    hb = G.uniform_rows(1500, 10, seed=16, m=2000)
    out["heavyrow64_f64"] = (ha, hb, np.float64)
    return out


def main(outdir: str) -> int:
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    manifest = {}
    for name, (A, B, dt) in cases().items():
        A = A.astype(dt)
        B = B.astype(dt)
        save_csr(out / f"{name}.A.csr", A)
        save_csr(out / f"{name}.B.csr", B)
        entry = {"dtype": np.dtype(dt).name, "m": A.m, "k": A.n, "n": B.n,
                 "nip": oracle.nip(A, B)}
        for which, fn in (("proposal", oracle.ref_proposal), ("cusparse2", oracle.ref_cusparse2)):
            try:
                C = fn(A, B, dt)
                save_csr(out / f"{name}.C_{which}.csr", C)
                entry[f"nnz_{which}"] = C.nnz
            except Exception as e:  # record, keep going
                entry[f"error_{which}"] = str(e)
        manifest[name] = entry
        print(name, entry, flush=True)
    (out / "manifest.json").write_text(json.dumps(manifest, indent=1))
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py OUTPUT_DIR")
    sys.exit(main(sys.argv[1]))
