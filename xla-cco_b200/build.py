"""Build libcco.so (the C-ABI CUDA library) in-tree for sm_100a.

    python xla-cco_b200/build.py            # incremental
    python xla-cco_b200/build.py --force    # rebuild

The library lands in ``xla-cco_b200/xla_cco/_lib/libcco.so`` next to the
Python package that loads it, so it travels with the source tree. nvcc
cross-compiles without a GPU; the CUDA runtime is linked statically.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent
REPO = PKG_ROOT.parent
CSRC = PKG_ROOT / "csrc"
INCLUDE = REPO / "include"
OUT_DIR = PKG_ROOT / "xla_cco" / "_lib"
LIB = OUT_DIR / "libcco.so"

SOURCES = ["cco_api.cu", "cco_eval.cu", "cco_opt.cu", "cco_relax.cu", "cco_serve.cu", "cco_flow.cu", "cco_md.cu", "cco_pairs.cu",
           "cco_hessian.cu", "cco_stepper.cu", "cco_persist.cu"]
HEADERS = ["cco_internal.cuh", "cco_opt.cuh", "cco_host.cuh", "cco_flow.cuh", "cco_md.cuh",
           "cco_eval_bodies.cuh", "cco_opt_bodies.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]  # fmt: skip


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [INCLUDE / "cco.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


PEAKS_LIB = OUT_DIR / "libcco_peaks.so"


def build_peaks(force: bool = False) -> Path:
    """Compile the FMA throughput probe (measurement utility used by bench.py)."""
    src = CSRC / "peaks.cu"
    if not force and PEAKS_LIB.exists() and PEAKS_LIB.stat().st_mtime > src.stat().st_mtime:
        return PEAKS_LIB
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", str(PEAKS_LIB), str(src)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libcco_peaks.so")
    return PEAKS_LIB


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile the library if any source is newer than it; return its path."""
    build_peaks(force)
    if not force and not _stale():
        return LIB
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, *(extra or []), "-shared", f"-I{INCLUDE}", f"-I{CSRC}",
           "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]  # fmt: skip
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libcco.so")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    args = ap.parse_args()
    extra = ["-Xptxas", "-v"] if args.ptxas_v else None
    print(build(force=args.force or args.ptxas_v, verbose=True, extra=extra))
