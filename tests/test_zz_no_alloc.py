"""pgpu_rates_noalloc (rates in a fixed static device scratch, no device
allocation by the library) against the context path (pgpu_solve +
pgpu_get_rates) on two calls in a row.

The file name sorts last so the test also runs after every other GPU test in
the same process; it passes alone as well.  Device buffers for the inputs and
outputs come from torch: they are the caller's memory, which is what this
entry point expects.
"""
import numpy as np
import pytest

from pawan_b200 import capi, cases

NU = 1e-4


def context_rates(w):
    # One target per thread, 256-source tiles and 8 source chunks: the launch
    # and chunking the no-allocation path uses for n <= 20000, so the two sums
    # are the same FP32 additions in the same order.
    with capi.Context(precision=capi.FP32C, nu=NU, block=256, tpt=1, chunks=8) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.solve()
        return c.rates(k)


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
    for w in (first, second):
        v, a = noalloc_rates(w)
        vr, ar = context_rates(w)
        assert np.all(np.isfinite(v)) and np.all(np.isfinite(a))
        np.testing.assert_array_equal(v, vr)
        np.testing.assert_array_equal(a, ar)
    # the same input again gives the same output (counters reset, no stale state)
    v2, a2 = noalloc_rates(second)
    np.testing.assert_array_equal(v2, v)
    np.testing.assert_array_equal(a2, a)


@pytest.mark.gpu
def test_noalloc_rejects_systems_above_its_capacity(gpu):
    n = capi.NOALLOC_MAX_N + 1
    with pytest.raises(capi.PgpuError, match="capacity of the fixed scratch array"):
        # rejected before any pointer is used
        capi.rates_noalloc(0, 0, 0, 0, n, NU, 0, 0)
