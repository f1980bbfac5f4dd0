"""Build liblogosq_b200.so (the CUDA engine) in-tree with nvcc for sm_100a.

Usage: python -m logosq_b200.build [--force]

The library is a plain C-ABI shared object; it links only the CUDA runtime
(and fetches cuTensorMapEncodeTiled from the driver at run time).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "liblogosq_b200.so"
BUILD = HERE / "_build"

SOURCES = [
    "api_state.cu",
    "gates.cu",
    "fused.cu",
    "variational.cu",
    "profile.cu",
    "batch.cu",
    "tc.cu",
    "learned.cu",
    "noise.cu",
]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-rdc=false",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = ([src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) +
            list((HERE.parent / "include").glob("*.h")))
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not OUT.exists() or any(o.stat().st_mtime > OUT.stat().st_mtime for o in objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
               *[str(o) for o in objs], "-o", str(OUT), "-lcudart_static", "-ldl", "-lrt",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
