"""Builds the sm_100a shared library of the B200 vortex-particle backend.

    python -m pawan_b200.build [--ptxas-verbose]

Compiles every ``csrc/*.cu`` with nvcc for ``sm_100a`` into
``pawan_b200/lib/libpawan_gpu.so`` (in-tree, so it travels with the
repository snapshot to the GPU machine).  No JIT and no fast-math: the
compensated FP32 accumulation relies on IEEE additions.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libpawan_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(ROOT / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [*CSRC.glob("*.cu"), *CSRC.glob("*.cuh"), *CSRC.glob("*.inc"), *(ROOT / "include").glob("*.h")]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objs = []
    tmp = LIBDIR / "_obj"
    tmp.mkdir(exist_ok=True)
    for src in sources():
        obj = tmp / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    out = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(out), *objs, "-lcudart"], check=True)
    os.replace(out, LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose_ptxas="--ptxas-verbose" in sys.argv)
    print(LIB)
