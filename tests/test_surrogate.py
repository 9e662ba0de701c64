"""Far-field surrogate: octree near field (exact) + multipole far field, with
the sampled-target gate that reverts to the direct sum."""
import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rings():
    return cases.leapfrog_rings(n_total=200_000)


def direct(w, nu=1e-4):
    c = capi.Context(precision=capi.FP32C, nu=nu)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.solve()
    v, a = c.rates(k)
    c.close()
    return v, a


def surrogate(w, nu=1e-4, **kw):
    c = capi.Context(precision=capi.FP32C, nu=nu)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.surrogate_enable(**kw)
    c.solve()
    v, a = c.rates(k)
    st = c.surrogate_stats()
    c.close()
    return v, a, st


def test_all_near_equals_direct(gpu, rings):
    """With a near field covering everything, every source is summed exactly
    once through the leaves: the result is the direct sum."""
    vd, ad = direct(rings)
    v, a, st = surrogate(rings, near_widths=1e9, check_targets=0)
    assert st["far_entries"] == 0 and st["leaves"] > 100
    # only the FP32 summation order differs from the direct kernel
    assert O.rel_err(v, vd) < 5e-6
    assert O.rel_err(a, ad) < 5e-6


def test_orders_converge_and_quadrupole_meets_gate(gpu, rings):
    vd, ad = direct(rings)
    errs, derrs = [], []
    for order in (0, 1, 2, 3):
        # four cube widths, where the truncation error is largest
        v, a, st = surrogate(rings, order=order, check_targets=0, near_widths=4.0)
        errs.append(O.rel_err(v, vd))
        derrs.append(O.rel_err(a, ad))
        assert st["fallbacks"] == 0
    print("velocity / dalpha errors by order:", [f"{e:.2e}/{d:.2e}" for e, d in zip(errs, derrs)])
    assert errs[2] < errs[0]
    assert errs[2] < 1e-4, errs
    # the octupole lowers both errors further
    assert errs[3] < errs[2] and derrs[3] < derrs[2], (errs, derrs)


def test_sampled_gate_reports_error(gpu, rings):
    vd, ad = direct(rings)
    v, a, st = surrogate(rings, order=2, tolerance=1.0)
    full = O.rel_err(v, vd)
    assert st["evaluations"] == 1 and st["fallbacks"] == 0
    # the sampled estimate is a lower bound of the full max-norm error, of the same size
    assert st["last_err_vel"] <= full * 1.0001 + 1e-12
    assert st["last_err_vel"] > 0.05 * full


def test_gate_reverts_to_direct_sum(gpu, rings):
    vd, ad = direct(rings)
    v, a, st = surrogate(rings, order=0, tolerance=1e-12)
    assert st["fallbacks"] == 1
    assert O.rel_err(v, vd) < 2e-6 and O.rel_err(a, ad) < 2e-6


def test_gate_also_reverts_on_dalpha_error(gpu, rings):
    """A tolerance between the sampled velocity error and the larger sampled
    dalpha/dt error: the velocity alone would pass, the stretching does not."""
    _, _, st = surrogate(rings, order=1, tolerance=1.0)
    ev, ea = st["last_err_vel"], st["last_err_dalpha"]
    assert ea > ev > 0
    vd, ad = direct(rings)
    v, a, st = surrogate(rings, order=1, tolerance=0.5 * (ev + ea))
    assert st["fallbacks"] == 1 and st["max_err_dalpha"] == st["last_err_dalpha"]
    assert O.rel_err(v, vd) < 2e-6 and O.rel_err(a, ad) < 2e-6


def test_surrogate_rk4_steps_track_direct(gpu):
    w = cases.leapfrog_rings(n_total=100_000)
    out = []
    for sur in (False, True):
        c = capi.Context(precision=capi.FP32C, nu=1e-4)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        if sur:
            c.surrogate_enable(order=2)
        c.step("rk4", 0.005, 2)
        out.append(c.state(k))
        if sur:
            assert c.surrogate_stats()["evaluations"] == 8
        c.close()
    assert O.rel_err(out[1][0] - w.pos, out[0][0] - w.pos) < 1e-4
    assert O.rel_err(out[1][1], out[0][1]) < 1e-4


def test_surrogate_host_errors(gpu):
    w = cases.ring_stations(stations=40)
    c = capi.Context(precision=capi.FP64, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    with pytest.raises(capi.PgpuError):
        c.surrogate_enable()
    c3 = capi.Context(precision=capi.FP32C, nu=1e-4)
    a = c3.add_wake(w.n, system=0)
    b = c3.add_wake(w.n, system=1)
    c3.set_particles(a, w)
    c3.set_particles(b, w)
    with pytest.raises(capi.PgpuError):
        c3.surrogate_enable()


def test_octree_partitions_particles(gpu):
    w = cases.leapfrog_rings(n_total=50_000)
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.surrogate_enable(check_targets=0, leaf_size=64)
    c.solve()
    t = c.surrogate_tree()
    assert np.array_equal(np.sort(t["idx"]), np.arange(w.n))
    cells = t["cells"]
    assert cells[0, 0] == 0 and cells[0, 1] == w.n
    for i, (s0, s1, fc, nc) in enumerate(cells):
        if nc:
            ch = cells[fc:fc + nc]
            assert ch[0, 0] == s0 and ch[-1, 1] == s1 and np.all(ch[1:, 0] == ch[:-1, 1])
    lv = cells[t["leaves"]]
    assert np.all(cells[t["leaves"], 3] == 0)
    order = np.argsort(lv[:, 0])
    assert lv[order[0], 0] == 0 and lv[order[-1], 1] == w.n and np.all(lv[order][1:, 0] == lv[order][:-1, 1])
    assert np.all(lv[:, 1] - lv[:, 0] <= 64)


@pytest.mark.parametrize("case", ["ring1m", "leapfrog1m"])
def test_surrogate_vs_fp64_restatement(gpu, case):
    """The quadrupole far field at 1M particles (the 1000 x 1000 ring with
    sigma = 0.02, and two coaxial leapfrogging rings) against the oracle's FP64 restatement of
    PAWAN's pair sum on 256 seeded targets: velocity and dalpha/dt both within
    the 1e-4 gate, with no fallback (so the surrogate's own result is what is
    compared)."""
    if case == "ring1m":
        w = cases.ring_gaussian(stations=1000, per_section=1000, sigma=0.02, seed=1)
    else:
        w = cases.leapfrog_rings(n_total=1_000_000)
    v, a, st = surrogate(w, order=2, tolerance=1e-4, check_targets=4096)
    assert st["fallbacks"] == 0, st
    rows = np.sort(np.random.default_rng(5).choice(w.n, 256, replace=False))
    vr, ar = O.restate_rates(w, 1e-4, targets=rows)
    ev, ea = O.rel_err(v[rows], vr), O.rel_err(a[rows], ar)
    print(f"{case}: surrogate vs FP64 restatement, velocity {ev:.2e}, dalpha/dt {ea:.2e}; sampled gate "
          f"{st['last_err_vel']:.2e} / {st['last_err_dalpha']:.2e}")
    assert ev <= 1e-4 and ea <= 1e-4
