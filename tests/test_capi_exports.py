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


@pytest.mark.parametrize("kw, msg", [({"precision": 7}, "unknown precision 7"),
                                     ({"kernel": 5}, "unknown regularisation kernel 5"),
                                     ({"block": 96}, "no compiled pair-kernel shape with block 96")])
def test_invalid_config_is_rejected_before_any_device_call(kw, msg):
    # the configuration is checked before pgpu_create touches a device, so
    # this runs without a GPU; the reason comes back through
    # pgpu_last_error(NULL)
    capi.load(build_if_missing=True)
    with pytest.raises(capi.PgpuError, match=msg) as e:
        capi.Context(**kw)
    assert e.value.code == capi.PGPU_EINVAL
