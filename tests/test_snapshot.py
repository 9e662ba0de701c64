"""Asynchronous state snapshots (pgpu_snapshot_begin / pgpu_snapshot_wait),
the download that feeds the per-step .wake records of PAWAN's offline loop
(__integration::integrate, integration.cpp:42-50).

A snapshot taken after step i and read while step i + 1 runs must hold the
state after step i bit for bit, as the synchronous pgpu_get_state gives it.
"""
from pathlib import Path

import numpy as np
import pytest

from pawan_b200 import capi, cases

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _twowake():
    g = np.load(GOLD / "twowake.npz")
    w1 = cases.Wake(g["pos1"], g["alpha1"], g["sigma1"], g["vol1"])
    w2 = cases.Wake(g["pos2"], g["alpha2"], g["sigma2"], g["vol2"])
    return float(g["nu"]), w1, w2


def _ctx(prec, nu, wakes, caps=None):
    c = capi.Context(precision=prec, nu=nu)
    ids = [c.add_wake(caps[i] if caps else w.n) for i, w in enumerate(wakes)]
    for i, w in zip(ids, wakes):
        c.set_particles(i, w)
    return c, ids


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32C])
@pytest.mark.parametrize("timing", [True, False])
def test_snapshots_equal_synchronous_state(gpu, prec, timing):
    nu, w1, w2 = _twowake()
    # the second wake has spare capacity: snapshots hold the live rows only
    a, ids = _ctx(prec, nu, [w1, w2], caps=[w1.n, w2.n + 300])
    b, idb = _ctx(prec, nu, [w1, w2], caps=[w1.n, w2.n + 300])
    a.set_timing(timing)
    ref = []
    for _ in range(5):
        b.step("rk4", 0.01, 1)
        ref.append([b.state(k) for k in idb])
    got = []
    for i in range(5):
        a.step("rk4", 0.01, 1)
        a.snapshot_begin(i % 2)
        if i:
            got.append(a.snapshot_wait((i - 1) % 2))  # read while step i runs
    got.append(a.snapshot_wait(4 % 2))
    a.sync()
    for i in range(5):
        assert len(got[i]) == 2
        for k in range(2):
            np.testing.assert_array_equal(got[i][k][0], ref[i][k][0])
            np.testing.assert_array_equal(got[i][k][1], ref[i][k][1])
    # the context's own state after the last step is the last snapshot
    for k in range(2):
        x, al = a.state(ids[k])
        np.testing.assert_array_equal(x, got[4][k][0])
        np.testing.assert_array_equal(al, got[4][k][1])
    a.close()
    b.close()


def test_snapshot_follows_growth_and_repeats(gpu):
    """A wake that grows between snapshots: each snapshot holds the rows live
    when it was begun; waiting twice on one slot returns the same data."""
    w = cases.ring_gaussian(stations=20, per_section=50, seed=3)
    extra = cases.ring_gaussian(stations=4, per_section=50, seed=4)
    with capi.Context(precision=capi.FP64, nu=1e-4) as c:
        k = c.add_wake(w.n + extra.n)
        c.set_particles(k, w)
        c.snapshot_begin(0)
        s0 = c.snapshot_wait(0)
        np.testing.assert_array_equal(s0[0][0], w.pos)
        np.testing.assert_array_equal(s0[0][1], w.alpha)
        c.append_particles(k, extra)
        c.snapshot_begin(1)
        s1 = c.snapshot_wait(1, timeout=30.0)
        assert s1[0][0].shape == (w.n + extra.n, 3)
        np.testing.assert_array_equal(s1[0][0][w.n:], extra.pos)
        again = c.snapshot_wait(1)
        np.testing.assert_array_equal(again[0][1], s1[0][1])


def test_snapshot_errors_and_watchdog(gpu):
    """Argument errors, and a wait with a short deadline behind a queued RK4
    step of a 400k ring: PGPU_ETIMEOUT, the copy still lands, the context
    stays usable."""
    w = cases.ring_gaussian(stations=400, per_section=1000, seed=1)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(w.n)
        with pytest.raises(capi.PgpuError) as e:
            c.snapshot_begin(0)  # nothing uploaded yet
        assert e.value.code == capi.PGPU_EINVAL
        c.set_particles(k, w)
        for bad in (-1, 2):
            with pytest.raises(capi.PgpuError) as e:
                c.snapshot_begin(bad)
            assert e.value.code == capi.PGPU_EINVAL
        with pytest.raises(capi.PgpuError) as e:
            c.snapshot_wait(1)  # never begun
        assert e.value.code == capi.PGPU_EINVAL
        c.set_timing(False)
        c.step("rk4", 0.005, 1)
        c.snapshot_begin(0)
        with pytest.raises(capi.PgpuError) as e:
            c.snapshot_wait(0, timeout=0.005)
        assert e.value.code == capi.PGPU_ETIMEOUT
        snap = c.snapshot_wait(0, timeout=60.0)
        c.sync()
        x, al = c.state(k)
        np.testing.assert_array_equal(snap[0][0], x)
        np.testing.assert_array_equal(snap[0][1], al)
