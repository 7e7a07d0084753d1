"""The fold's host-side chunking (fold_chunks / fold_chunk_list in
fbls_b200/csrc/fold.cu), checked on the CPU through the built library:
tests/host_logic/fold_chunks_check.cpp links it and checks the properties
the walking fold relies on (a chunk's cells are distinct bins at every
period of the launch; chunks tile the observations) and that the list sized
by the chunk-count bound equals the chunking into a buffer of n + 2."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

from fbls_b200 import _native

CHECK = Path(__file__).resolve().parent / "host_logic" / "fold_chunks_check.cpp"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def test_fold_chunk_list_equals_the_full_buffer_and_keeps_the_limits(tmp_path):
    lib_dir = _native.LIB_PATH.parent
    exe = tmp_path / "fold_chunks_check"
    build = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", str(CHECK),
                            f"-L{lib_dir}", "-lfbls_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    out = json.loads(run.stdout.strip().splitlines()[-1])
    assert out["cases"] == 2000
    assert out["bad_equal"] == 0 and out["bad_cover"] == 0 and out["bad_limits"] == 0 and out["bad_ends"] == 0
    # the buffer follows the chunk count, not n (here a seventh of n + 2 in all)
    assert out["bound_over_full"] < 0.5
