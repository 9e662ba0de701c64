"""GPU parity: the sm_100a path through the C ABI vs PAWAN's own code.

Gates: FP64 mode within 1e-10 and FP32-compensated mode within 1e-5
(max-norm relative error, max_i |x_i - ref_i| / max_i |ref_i|), both against
PAWAN's compiled CPU code or the golden fixtures it produced.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
TOL = {capi.FP64: 1e-10, capi.FP32C: 1e-5}
PREC = [capi.FP64, capi.FP32C]


def golden_wake(name="ring1000.npz"):
    g = np.load(GOLD / name)
    return g, cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])


def ctx_with(wakes, precision, nu, systems=None, capacity=None, **kw):
    c = capi.Context(precision=precision, nu=nu, **kw)
    ids = []
    for i, w in enumerate(wakes):
        ids.append(c.add_wake(capacity[i] if capacity else w.n, systems[i] if systems else 0))
    for i, w in zip(ids, wakes):
        c.set_particles(i, w)
    return c, ids


@pytest.mark.parametrize("prec", PREC)
def test_rates_vs_golden(gpu, prec):
    g, w = golden_wake()
    c, _ = ctx_with([w], prec, float(g["nu"]))
    c.solve()
    v, a = c.rates(0)
    assert O.rel_err(v, g["vel"]) < TOL[prec]
    assert O.rel_err(a, g["dalpha"]) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
def test_rates_ring5000_sampled(gpu, prec):
    g = np.load(GOLD / "ring5000.npz")
    w = cases.ring_stations()
    c, _ = ctx_with([w], prec, float(g["nu"]))
    c.solve()
    v, a = c.rates(0)
    rows = g["rows"]
    assert O.rel_err(v[rows], g["vel"]) < TOL[prec]
    assert O.rel_err(a[rows], g["dalpha"]) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_steps_vs_golden(gpu, prec, scheme):
    g, w = golden_wake()
    c, _ = ctx_with([w], prec, float(g["nu"]))
    c.step(scheme, float(g["dt"]), 2)
    c.sync()
    x, al = c.state(0)
    assert O.rel_err(x, g[f"{scheme}_pos"]) < TOL[prec]
    assert O.rel_err(al, g[f"{scheme}_alpha"]) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
def test_rk4_step_ring5000_sampled(gpu, prec):
    g = np.load(GOLD / "ring5000.npz")
    w = cases.ring_stations()
    c, _ = ctx_with([w], prec, float(g["nu"]))
    c.step("rk4", float(g["dt"]), 1)
    x, al = c.state(0)
    rows = g["rows"]
    assert O.rel_err(x[rows], g["rk4_pos"]) < TOL[prec]
    assert O.rel_err(al[rows], g["rk4_alpha"]) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
def test_euler_vs_reference(gpu, ref_available, prec):
    _, w = golden_wake()
    R = O.RefSystem([w], 1e-4)
    R.step("euler", 0.01, 3)
    xr, ar = R.state()
    c, _ = ctx_with([w], prec, 1e-4)
    c.step("euler", 0.01, 3)
    x, al = c.state(0)
    assert O.rel_err(x, xr) < TOL[prec]
    assert O.rel_err(al, ar) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
def test_two_wakes_one_system(gpu, prec):
    g = np.load(GOLD / "twowake.npz")
    w1 = cases.Wake(g["pos1"], g["alpha1"], g["sigma1"], g["vol1"])
    w2 = cases.Wake(g["pos2"], g["alpha2"], g["sigma2"], g["vol2"])
    c, ids = ctx_with([w1, w2], prec, float(g["nu"]))
    c.solve()
    v1, d1 = c.rates(ids[0])
    v2, d2 = c.rates(ids[1])
    assert O.rel_err(np.concatenate([v1, v2]), np.concatenate([g["vel1"], g["vel2"]])) < TOL[prec]
    assert O.rel_err(np.concatenate([d1, d2]), np.concatenate([g["dalpha1"], g["dalpha2"]])) < TOL[prec]
    d, _ = c.diagnose(0)
    ref = g["diag"]
    tol = 1e-9 if prec == capi.FP64 else 1e-4
    np.testing.assert_allclose(d[3:14], ref[3:14], rtol=tol, atol=tol * np.abs(ref[3:14]).max())


@pytest.mark.parametrize("prec", PREC)
def test_diagnostics_vs_golden(gpu, prec):
    g, w = golden_wake()
    c, _ = ctx_with([w], prec, float(g["nu"]))
    d, vbi = c.diagnose(0)
    ref = g["diag"]
    # O(N) sums are FP64 in both modes
    np.testing.assert_allclose(d[3:9], ref[3:9], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(vbi, g["vbi"], rtol=1e-10, atol=1e-14)
    assert d[10] == 0.0 and d[11] == 0.0
    tol = 1e-10 if prec == capi.FP64 else 1e-5
    np.testing.assert_allclose(d[12:14], ref[12:14], rtol=tol)
    # helicity of a planar ring is a cancelling sum: compare against its scale
    assert abs(d[9] - ref[9]) < tol * max(abs(ref[9]), 1e-3 * ref[12])
    assert abs(d[14] - ref[14]) < 1e-9


@pytest.mark.parametrize("prec", PREC)
def test_batched_systems_equal_separate(gpu, prec):
    """Independent systems in one launch give the same rates as one context each."""
    # at least 16 stations per ring: with fewer, strengths are (anti)parallel,
    # true stretching vanishes and only input rounding is left to compare
    rings = cases.uneven_rings(count=6, nmin=400, nmax=4000, seed=7)
    c, ids = ctx_with(rings, prec, 1e-4, systems=list(range(len(rings))))
    c.solve()
    for i, w in zip(ids, rings):
        v, a = c.rates(i)
        vr, ar = O.restate_rates(w, 1e-4)
        assert O.rel_err(v, vr) < TOL[prec]
        assert O.rel_err(a, ar) < TOL[prec]


@pytest.mark.parametrize("shape", [(128, 1), (128, 2), (256, 1), (256, 2), (64, 2), (128, 4)])
def test_every_kernel_shape(gpu, shape):
    g, w = golden_wake()
    c, _ = ctx_with([w], capi.FP32C, float(g["nu"]), block=shape[0], tpt=shape[1])
    c.solve()
    v, a = c.rates(0)
    assert O.rel_err(v, g["vel"]) < 1e-5
    assert O.rel_err(a, g["dalpha"]) < 1e-5


def test_graph_and_eager_steps_identical(gpu):
    _, w = golden_wake()
    out = []
    for graphs in (True, False):
        c, _ = ctx_with([w], capi.FP32C, 1e-4, use_graphs=graphs)
        c.step("rk4", 0.01, 3)
        out.append(c.state(0))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("n", [1, 2, 31, 255, 257, 1025])
def test_ragged_sizes(gpu, n):
    _, w = golden_wake()
    ws = w.subset(n)
    c, _ = ctx_with([ws], capi.FP64, 1e-4, capacity=[n + 100])
    c.solve()
    v, a = c.rates(0)
    vr, ar = O.restate_rates(ws, 1e-4)
    if n == 1:
        assert np.all(v == 0) and np.all(a == 0)
    else:
        assert O.rel_err(v, vr) < 1e-10 and O.rel_err(a, ar) < 1e-10


def test_empty_wake_and_growth(gpu):
    _, w = golden_wake()
    c = capi.Context(precision=capi.FP64, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w.subset(0))
    c.solve()
    c.step("rk4", 0.01, 1)
    assert c.num_particles(k) == 0
    c.append_particles(k, w.subset(400))
    rest = cases.Wake(w.pos[400:], w.alpha[400:], w.sigma[400:], w.vol[400:])
    c.append_particles(k, rest)
    c.solve()
    v, a = c.rates(k)
    g = np.load(GOLD / "ring1000.npz")
    assert O.rel_err(v, g["vel"]) < 1e-10 and O.rel_err(a, g["dalpha"]) < 1e-10


def test_host_errors(gpu):
    _, w = golden_wake()
    c = capi.Context()
    k = c.add_wake(10)
    with pytest.raises(capi.PgpuError) as e:
        c.set_particles(k, w.subset(11))
    assert e.value.code == capi.PGPU_EINVAL
    c.set_particles(k, w.subset(10))
    with pytest.raises(capi.PgpuError):
        c.add_wake(5)
    with pytest.raises(capi.PgpuError):
        c.step("rk4", 0.01, -1)
    with pytest.raises(capi.PgpuError):
        c.rates(3)


def test_non_finite_state_is_reported(gpu):
    _, w = golden_wake()
    bad = w.copy()
    bad.alpha[5, 0] = np.nan
    c, _ = ctx_with([bad], capi.FP32C, 1e-4)
    c.step("euler", 0.01, 1)
    with pytest.raises(capi.PgpuError) as e:
        c.sync()
    assert e.value.code == capi.PGPU_ENUMERIC


def test_flat_state_roundtrip(gpu):
    g, w = golden_wake()
    c, _ = ctx_with([w], capi.FP64, 1e-4)
    maxn = [1200]
    st = c.get_states_flat(maxn)
    np.testing.assert_array_equal(st[:3000].reshape(-1, 3), w.pos)
    np.testing.assert_array_equal(st[3600:6600].reshape(-1, 3), w.alpha)
    c.set_states_flat(st, maxn)
    c.solve()
    r = c.get_rates_flat(maxn)
    assert O.rel_err(r[:3000].reshape(-1, 3), g["vel"]) < 1e-10


def test_probe_matches_reference_getvi(gpu, ref_available):
    _, w = golden_wake()
    R = O.RefSystem([w], 1e-4)
    pts = np.array([[0.0, 0.0, 0.0], [0.0, 0.8, 0.0], [-0.255, 0.8, 0.02], [1.0, 0.0, 0.1], [2.0, 1.0, -0.5]])
    ref = np.array([R.getvi(p) for p in pts])
    c, _ = ctx_with([w], capi.FP64, 1e-4)
    v = c.probe(pts)
    assert O.rel_err(v, ref) < 1e-10


@pytest.mark.parametrize("prec", PREC)
def test_inflow_operator_split(gpu, prec):
    """x += vinf dt after every step (updateVinfEffect, wake.cpp:564-577): a uniform
    shift leaves the interaction unchanged, so the state is the no-inflow state
    moved by vinf * t."""
    _, w = golden_wake()
    vinf = (0.01, -0.02, -0.05)
    out = []
    for v in ((0.0, 0.0, 0.0), vinf):
        c, _ = ctx_with([w], prec, 1e-4, vinf=v)
        c.step("rk3", 0.01, 4)
        out.append(c.state(0))
    # FP32C rounds the shifted positions differently, so only FP64 is exact to rounding
    atol = 1e-12 if prec == capi.FP64 else 1e-6
    np.testing.assert_allclose(out[1][0] - out[0][0], np.tile(np.array(vinf) * 0.04, (w.n, 1)), atol=atol)
    assert O.rel_err(out[1][1], out[0][1]) < TOL[prec]


@pytest.mark.parametrize("prec", PREC)
def test_growing_wake_matches_restatement(gpu, prec):
    """A wake that gains particles between RK3 steps (the growing rotor wake)
    replays the same captured step graph and matches the FP64 restatement
    stepping the same sequence."""
    sh = cases.RotorShedder(per_blade=40)
    c = capi.Context(precision=prec, nu=1e-4)
    k = c.add_wake(4 * 40 * 6)
    c.set_particles(k, sh.shed())
    first = cases.RotorShedder(per_blade=40)
    w_ref = first.shed()
    for it in range(5):
        c.step("rk3", sh.dt, 1)
        x, al = O.restate_step(w_ref, 1e-4, "rk3", sh.dt, 1)
        w_ref = cases.Wake(x, al, w_ref.sigma, w_ref.vol)
        new = sh.shed()
        first.shed()
        c.append_particles(k, new)
        w_ref = cases.Wake.concat([w_ref, new])
    x, al = c.state(k)
    assert x.shape[0] == w_ref.n == 4 * 40 * 6
    assert O.rel_err(x, w_ref.pos) < TOL[prec]
    assert O.rel_err(al, w_ref.alpha) < TOL[prec]


@pytest.fixture(scope="module")
def ring1m():
    """The 1M-particle ring: 1000 stations x 1000 particles, Gaussian
    cross-section, sigma = 0.02, seed 1."""
    return cases.ring_gaussian()


@pytest.fixture(scope="module")
def ring1m_rates(ring1m):
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(ring1m.n)
        c.set_particles(k, ring1m)
        c.solve()
        return c.rates(k)


def test_rates_ring1m_sampled_vs_fp64_restatement(gpu, ring1m, ring1m_rates):
    """FP32C at N = 1M on 256 seeded targets against the FP64 restatement of
    PAWAN's pair sum (gate 1e-5)."""
    v, a = ring1m_rates
    rows = np.sort(np.random.default_rng(11).choice(ring1m.n, 256, replace=False))
    vr, ar = O.restate_rates(ring1m, 1e-4, targets=rows)
    ev, ea = O.rel_err(v[rows], vr), O.rel_err(a[rows], ar)
    print(f"1M ring, 256 sampled targets: velocity {ev:.2e}, dalpha/dt {ea:.2e}")
    assert ev < TOL[capi.FP32C] and ea < TOL[capi.FP32C]


def test_ring1m_stretching_and_diffusion_sum_to_zero(gpu, ring1m_rates):
    """Size-independent check at N = 1M: the transpose-scheme stretching and
    the diffusion of an ordered pair are antisymmetric (interaction_utils.h:
    492-495, 358-369), so sum_i dalpha_i/dt vanishes up to rounding."""
    _, a = ring1m_rates
    tot = np.abs(a.sum(axis=0)).max()
    scale = np.abs(a).sum(axis=0).max()
    print(f"1M ring: |sum dalpha/dt| / sum |dalpha/dt| = {tot / scale:.2e}")
    assert tot <= 1e-6 * scale


def test_64_uneven_rings_batched_sampled(gpu):
    """64 independent rings, N log-uniform in
    [2e3, 2e5] (seed 2), as 64 systems of one context evaluated in one
    persistent launch; 64 seeded targets of the three smallest and three
    largest rings against the FP64 restatement of each ring alone."""
    ws = cases.uneven_rings(count=64, nmin=2e3, nmax=2e5, seed=2)
    c, ids = ctx_with(ws, capi.FP32C, 1e-4, systems=list(range(len(ws))))
    c.solve()
    order = np.argsort([w.n for w in ws])
    rng = np.random.default_rng(3)
    worst = 0.0
    for i in list(order[:3]) + list(order[-3:]):
        w = ws[i]
        v, a = c.rates(ids[i])
        rows = np.sort(rng.choice(w.n, 64, replace=False))
        vr, ar = O.restate_rates(w, 1e-4, targets=rows)
        worst = max(worst, O.rel_err(v[rows], vr), O.rel_err(a[rows], ar))
    c.close()
    print(f"64 rings, {sum(w.n for w in ws)} particles: worst sampled error {worst:.2e}")
    assert worst < TOL[capi.FP32C]


def test_conservation_and_fp32c_trajectory(gpu):
    """Ten RK4 steps of a 20k ring in both modes: total vorticity stays at
    rounding level and the FP32C trajectory follows the FP64 one within the
    FP32C gate."""
    from pawan_b200 import conservation
    res = conservation.run(stations=20, steps=10, every=5)
    last = res["records"][-1]
    print(conservation.markdown(res))
    assert last["fp64"]["total vorticity"] < 1e-13
    assert last["fp32c"]["total vorticity"] < 1e-9
    assert last["fp32c_vs_fp64"]["displacement"] < TOL[capi.FP32C]
    assert last["fp32c_vs_fp64"]["alpha"] < TOL[capi.FP32C]


def test_watchdog_times_out_and_work_completes(gpu):
    """Host-side failure detection: a sync with a short deadline on a queued
    RK4 step of a 400k ring returns PGPU_ETIMEOUT without disturbing the work;
    the next plain sync waits for it and the context stays usable."""
    w = cases.ring_gaussian(stations=400, per_section=1000, seed=1)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.set_timing(False)  # the step only queues its work
        c.step("rk4", 0.005, 1)
        with pytest.raises(capi.PgpuError) as e:
            c.sync(timeout=0.01)
        assert e.value.code == capi.PGPU_ETIMEOUT
        c.sync()
        c.sync(timeout=60.0)
        pos, _ = c.state(k)
        assert np.all(np.isfinite(pos))


def test_device_allocation_failure_is_reported(gpu):
    """A context whose capacity cannot be allocated (2^31 - 1 particles, about
    2 TB) fails with PGPU_ENOMEM at the first upload, frees what it got, and
    a normal context works afterwards."""
    w = cases.ring_stations(stations=40)
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(2 ** 31 - 1)
    with pytest.raises(capi.PgpuError) as e:
        c.set_particles(k, w)
    assert e.value.code == capi.PGPU_ENOMEM
    c.close()
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c2:
        k2 = c2.add_wake(w.n)
        c2.set_particles(k2, w)
        c2.solve()
        v, _ = c2.rates(k2)
        assert np.all(np.isfinite(v))


@pytest.mark.parametrize("prec", PREC)
def test_vorticity_field_vs_pawan_influence(gpu, ref_available, prec):
    """pgpu_influence on two interacting wakes of one system against PAWAN's
    own resolve()/influence() (interaction.cpp:59-62, 212-260)."""
    w1 = cases.ring_stations(stations=40, seed=0)
    w2 = cases.ring_stations(stations=30, R=0.7, seed=1)
    with O.quiet():
        R = O.RefSystem([w1, w2], 1e-4)
        kref = R.vorticity_field()
        R.close()
    c, ids = ctx_with([w1, w2], prec, 1e-4)
    k = np.vstack([c.vorticity_field(ids[0]), c.vorticity_field(ids[1])])
    c.close()
    assert O.rel_err(k, kref) < TOL[capi.FP64]  # FP64 in both modes


def test_vorticity_field_separate_systems_and_1m_sampled(gpu):
    """Systems do not see each other's particles; at N = 1M (an FP32C context;
    the field is FP64 in both modes) 256 seeded targets match the FP64
    restatement within the FP64 gate."""
    w1 = cases.ring_stations(stations=40, seed=0)
    w2 = cases.ring_stations(stations=30, R=0.7, seed=1)
    c, ids = ctx_with([w1, w2], capi.FP32C, 1e-4, systems=[0, 1])
    k1, k2 = c.vorticity_field(ids[0]), c.vorticity_field(ids[1])
    c.close()
    assert O.rel_err(k1, O.restate_vorticity_field(w1)) < TOL[capi.FP64]
    assert O.rel_err(k2, O.restate_vorticity_field(w2)) < TOL[capi.FP64]
    w = cases.ring_gaussian()
    c, ids = ctx_with([w], capi.FP32C, 1e-4)
    k = c.vorticity_field(ids[0])
    c.close()
    rows = np.sort(np.random.default_rng(13).choice(w.n, 256, replace=False))
    e = O.rel_err(k[rows], O.restate_vorticity_field(w, targets=rows))
    print(f"1M ring vorticity field, 256 sampled targets: {e:.2e}")
    assert e < TOL[capi.FP64]
