"""The C-ABI library loads and exports every entry point include/pawan_gpu.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

from pawan_b200 import build, capi

ROOT = Path(__file__).resolve().parents[1]


def declared():
    txt = (ROOT / "include" / "pawan_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(pgpu_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert sorted(capi.EXPORTS) == declared()


def test_library_exports_every_symbol():
    if not build.LIB.exists():
        build.build()
    lib = ctypes.CDLL(str(build.LIB))
    for name in declared():
        assert hasattr(lib, name), name


def test_version_and_shapes_without_gpu():
    lib = capi.load(build_if_missing=True)
    assert b"sm_100a" in lib.pgpu_version()
    shapes = capi.kernel_shapes()
    assert (256, 2) in shapes and len(shapes) >= 4
