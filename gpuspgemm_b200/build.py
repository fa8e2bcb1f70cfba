"""Build the native library in-tree: gpuspgemm_b200/libspgemm_b200.so.

Every CUDA source is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked with the static CUDA
runtime, so the library loads (dlopen) on a machine without a GPU driver and
the per-kernel ``.so`` is the one the tests and the bench load.

Usage: ``python -m gpuspgemm_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OBJ_DIR = PKG / "_build"
LIB = PKG / "libspgemm_b200.so"
# the CLI driver, one binary per value type (the reference picks the type at
# build time with USE_DOUBLE_PRECISION, cmake/options.cmake:2-3)
APPS = {PKG / "spgemm_app": ["-DUSE_DOUBLE_PRECISION"], PKG / "spgemm_app_f32": []}

SOURCES = ["k_bin.cu", "k_sym1.cu", "k_s2n.cu", "k_batch.cu", "k_transpose.cu", "spgemm.cu",
           "noalloc.cu"]
APP_SOURCES = ["app/spgemm_app.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "-Xptxas",
    "-warn-spills",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
    return path


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, flush=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile and link the library if any source is newer than it."""
    OBJ_DIR.mkdir(exist_ok=True)
    headers = _headers()
    jobs = []
    for name in SOURCES:
        src = CSRC / name
        obj = OBJ_DIR / (Path(name).stem + ".o")
        if force or _stale(obj, [src, *headers]):
            jobs.append((src, obj))
    if jobs:
        workers = min(len(jobs), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=workers) as ex:
            futs = [ex.submit(_compile, s, o, verbose) for s, o in jobs]
            for f in futs:
                f.result()
    objs = [OBJ_DIR / (Path(n).stem + ".o") for n in SOURCES]
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    _build_app(force)
    return LIB


def _build_app(force: bool) -> None:
    """The reference-compatible CLI driver (validate / save / benchmark)."""
    srcs = [CSRC / s for s in APP_SOURCES]
    if not all(s.exists() for s in srcs):
        return
    deps = [*srcs, *_headers(), LIB]
    for app, defs in APPS.items():
        if not (force or _stale(app, deps)):
            continue
        cmd = [
            nvcc(),
            *ARCH,
            "-O2",
            "-std=c++17",
            *defs,
            f"-I{INCLUDE}",
            f"-I{CSRC}",
            *map(str, srcs),
            "-o",
            str(app),
            f"-L{PKG}",
            "-lspgemm_b200",
            "-lcusparse",
            "-Xlinker",
            "-rpath,$ORIGIN",
        ]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"app build failed:\n{res.stdout}\n{res.stderr}")


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    lib = build(force=args.force, verbose=args.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
