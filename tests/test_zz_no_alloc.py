"""pgpu_rates_noalloc (rates in a fixed static device scratch, no device
allocation by the library) against the context path (pgpu_solve +
pgpu_get_rates) on two calls in a row, and against the oracle's FP64
restatement on sampled targets.

The file name sorts last so the test also runs after every other GPU test in
the same process; it passes alone as well.  Device buffers for the inputs and
outputs come from torch: they are the caller's memory, which is what this
entry point expects.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

NU = 1e-4
FP32C_GATE = 1e-5  # max-norm relative error of FP32C rates against FP64


def context_rates(w):
    # One target per thread, 256-source tiles and 8 source chunks: the launch
    # and chunking the no-allocation path uses for n <= 20000 on a GPU with at
    # least 139 resident pair-kernel CTAs, so the two sums are then the same
    # FP32 additions in the same order.
    with capi.Context(precision=capi.FP32C, nu=NU, block=256, tpt=1, chunks=8) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.solve()
        return c.rates(k)


def same_chunking() -> bool:
    """True when the no-allocation path splits a system of <= 20000 particles
    (at most 79 tiles of 256) into 8 source chunks, as context_rates does:
    it takes ceil(4 x resident CTAs / tiles) chunks, at most 8, and a GPU has
    at least one resident CTA per SM."""
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count >= 139


def noalloc_rates(w):
    import torch
    dev = torch.device("cuda:0")
    t = {f: torch.from_numpy(np.ascontiguousarray(getattr(w, f))).to(dev) for f in ("pos", "alpha", "sigma", "vol")}
    # NaN-filled outputs: every element must be written by the call
    vel = torch.full((w.n, 3), float("nan"), dtype=torch.float64, device=dev)
    dal = torch.full((w.n, 3), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    capi.rates_noalloc(t["pos"].data_ptr(), t["alpha"].data_ptr(), t["sigma"].data_ptr(), t["vol"].data_ptr(), w.n,
                       NU, vel.data_ptr(), dal.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    return vel.cpu().numpy(), dal.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_context_path_on_consecutive_calls(gpu):
    # a larger system, then a smaller one: the second call must not see any
    # of the first call's records or partials left in the scratch array
    first = cases.ring_gaussian(stations=40, per_section=500, seed=3)  # 20000
    second = cases.uneven_rings(count=1, nmin=6000, nmax=6000, seed=5)[0]
    assert first.n <= 20000 and second.n < first.n
    bitwise = same_chunking()
    for w in (first, second):
        v, a = noalloc_rates(w)
        vr, ar = context_rates(w)
        assert np.all(np.isfinite(v)) and np.all(np.isfinite(a))
        if bitwise:
            np.testing.assert_array_equal(v, vr)
            np.testing.assert_array_equal(a, ar)
        else:
            # another chunking only reorders the FP32 group sums
            assert O.rel_err(v, vr) < 1e-6 and O.rel_err(a, ar) < 1e-6
    # the same input again gives the same output (counters reset, no stale state)
    v2, a2 = noalloc_rates(second)
    np.testing.assert_array_equal(v2, v)
    np.testing.assert_array_equal(a2, a)


@pytest.mark.gpu
def test_noalloc_matches_fp64_restatement(gpu):
    w = cases.ring_gaussian(stations=32, per_section=1000, seed=7)  # 32000, close to the capacity
    assert w.n <= capi.NOALLOC_MAX_N
    rows = np.sort(np.random.default_rng(11).choice(w.n, 256, replace=False))
    vr, ar = O.restate_rates(w, NU, targets=rows)
    for _ in range(2):
        v, a = noalloc_rates(w)
        ev, ea = O.rel_err(v[rows], vr), O.rel_err(a[rows], ar)
        assert ev < FP32C_GATE and ea < FP32C_GATE, (ev, ea)


@pytest.mark.gpu
def test_noalloc_rejects_systems_above_its_capacity(gpu):
    n = capi.NOALLOC_MAX_N + 1
    with pytest.raises(capi.PgpuError, match="capacity of the fixed scratch array"):
        # rejected before any pointer is used
        capi.rates_noalloc(0, 0, 0, 0, n, NU, 0, 0)
