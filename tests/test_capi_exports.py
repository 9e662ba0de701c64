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


def test_wake_arrays_reject_short_arrays():
    # the library reads 3n, 3n, n and n values: a short array would be
    # over-read on the host, so the binding refuses it before any call
    import numpy as np

    from pawan_b200 import cases
    w = cases.ring_stations(stations=8, seed=0)
    arr = capi.wake_arrays(w)
    assert [a.size for a in arr] == [3 * w.n, 3 * w.n, w.n, w.n]
    assert all(a.dtype == np.float64 and a.flags.c_contiguous for a in arr)
    # contiguous FP64 input is passed through without a copy
    assert arr[0] is w.pos or np.shares_memory(arr[0], w.pos)
    short = cases.Wake(w.pos, w.alpha, w.sigma[:-1], w.vol)
    with pytest.raises(ValueError, match="sigma holds"):
        capi.wake_arrays(short)
    with pytest.raises(ValueError, match="alpha holds"):
        capi.wake_arrays(cases.Wake(w.pos, w.alpha[:-1], w.sigma, w.vol))


def test_surrogate_config_defaults_and_unknown_settings():
    # pgpu_surrogate_config_default is host-only: no GPU needed
    cfg = capi.surrogate_config(order=3, near_widths=4.5)
    assert cfg.order == 3 and cfg.near_widths == 4.5
    assert cfg.tolerance == 1e-4 and cfg.leaf_size == 256 and cfg.check_targets == 4096
    with pytest.raises(TypeError, match="unknown surrogate setting 'near_width'"):
        capi.surrogate_config(near_width=4.0)


def test_network_rows_are_checked():
    # the network reads rows x 24 features and rows x 6 targets
    import numpy as np
    x = capi._rows(np.zeros((5, 24)), capi.MLP_IN, "x")
    assert x.dtype == np.float32 and x.shape == (5, 24)
    with pytest.raises(ValueError, match=r"x must have shape \(rows, 24\)"):
        capi._rows(np.zeros((5, 20)), capi.MLP_IN, "x")
    with pytest.raises(ValueError, match="must have shape"):
        capi._rows(np.zeros(24), capi.MLP_IN, "x")
