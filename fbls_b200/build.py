"""Builds the fbls_b200 native library in-tree: fbls_b200/lib/libfbls_b200.so.

Every CUDA source is compiled for sm_100a only, with --fmad=false: the bin
index floor(t * scale), the template widths and the f32 pre-ranking merit must
round each multiply and add separately, as the reference's arithmetic does.
Host C++ is compiled with -ffp-contract=off for the same reason.

    python -m fbls_b200.build          # build (incremental by mtime)
    python -m fbls_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libfbls_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
              "-Xptxas", "-O3"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]

CU_SOURCES = ["fold.cu", "scan_kernels.cu", "evidence.cu", "proposal.cu", "rescore.cu", "biweight.cu", "cnn.cu", "host.cu", "host_maps.cu", "host_next.cu",
              "static_entry.cu", "precision.cu"]
CPP_SOURCES = ["prep.cpp"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else (shutil.which("nvcc") or "nvcc")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... (exit {res.returncode})")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles the CUDA and C++ sources and links the shared library."""
    BUILD.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    headers = _headers()
    objects = []
    nvcc = _nvcc()
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        if force or _stale(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)], verbose)
        objects.append(o)
    cxx = os.environ.get("CXX", shutil.which("g++") or "g++")
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        if force or _stale(o, [s] + headers):
            _run([cxx, *CXX_FLAGS, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)], verbose)
        objects.append(o)
    if force or _stale(LIB, objects):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objects), "-lcudart_static", "-lrt", "-ldl",
              "-lpthread"], verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", "-v", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print registers / spills per kernel")
    args = ap.parse_args()
    lib = build(force=args.force, verbose=args.verbose, ptxas_verbose=args.ptxas)
    print(lib)


if __name__ == "__main__":
    main()
