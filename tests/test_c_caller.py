"""The header is plain C: a C99 program (tests/c_abi_check.c) compiles
against include/pawan_gpu.h with -pedantic -Werror, links the library and
runs the entry points that need no GPU (CPU only)."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

from pawan_b200 import build

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c99_caller_builds_and_runs(tmp_path):
    if not build.LIB.exists():
        build.build()
    exe = tmp_path / "c_abi_check"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "c_abi_check.c"), "-o", str(exe), "-L", str(build.LIBDIR), "-lpawan_gpu",
                    f"-Wl,-rpath,{build.LIBDIR}"], check=True)
    # the library's CUDA runtime (libcudart.so.12) is found through the
    # environment's library path, as for the Python tests
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=dict(os.environ), timeout=60)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "sm_100a" in r.stdout
