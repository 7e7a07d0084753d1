"""The C ABI from C: tests/c_abi/abi_harness.c is compiled with gcc as C11
against include/fbls_b200.h and linked to the built library, as a foreign
host would link it, and run; the header also compiles as C++17. No GPU
calls succeed here (context creation must fail cleanly without a device)."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

import oracle
from fbls_b200 import _native

ROOT = Path(__file__).resolve().parent.parent
HARNESS = Path(__file__).resolve().parent / "c_abi" / "abi_harness.c"
INCLUDE = ROOT / "include"

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                                reason="needs gcc and g++")


def _cuda_visible() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_header_compiles_as_c_and_cxx(tmp_path):
    for cmd in (["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-fsyntax-only", "-x", "c"],
                ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c++"]):
        subprocess.run(cmd + [str(INCLUDE / "fbls_b200.h")], check=True, capture_output=True, text=True)


def test_c_harness_links_and_passes(tmp_path):
    lib_dir = _native.LIB_PATH.parent
    exe = tmp_path / "abi_harness"
    build = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{INCLUDE}", str(HARNESS),
                            f"-L{lib_dir}", "-lfbls_b200", f"-Wl,-rpath,{lib_dir}", "-lm", "-o", str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    out = json.loads(run.stdout.strip().splitlines()[-1])
    assert out["fails"] == 0
    assert out["version"].startswith("fbls_b200")
    assert out["grid_count"] == len(oracle.period_grid(0.5, 20.0, 50.0, 0.02, 3.0))
    assert out["data_error"] == "insufficient usable observations"
    if not _cuda_visible():
        assert out["device"] == 0 and out["create_status"] == 2  # FBLS_ERR_CUDA
