"""PAWAN's particle merge (__wake::merge, src/wake/wake.cpp:112-159), the
O(N^2) half of the relaxation of the coupled time loop.

Oracle: PAWAN's own merge (oracle/_ref/libpawanref.so, ref_merge) and the
grid-based restatement rs_merge (oracle/restate.c), pinned to it bit for bit.
The GPU path (pgpu_merge: candidate search on the device, PAWAN's sequential
loop replayed on the host) must reproduce both bit for bit: the merge makes
threshold decisions, so anything short of the same arithmetic could merge a
different set of particles.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

STEP = 100  # stepnum of the merge call; cases.merge_clusters ages are set for it


def pawan_merge(w, active):
    with O.quiet():
        R = O.RefSystem([w], 1e-4)
        R.merge(0, active, STEP)
        out = R.particles(0)
        R.close()
    return out


# ---------------------------------------------------------------- oracle (CPU)

@pytest.mark.parametrize("seed", [0, 1, 2])
def test_restated_merge_matches_pawan(ref_available, seed):
    w, n_elig, active = cases.merge_clusters(seed=seed)
    x, a, _, v = pawan_merge(w, active)
    xr, ar, vr, m = O.restate_merge(w, n_elig)
    assert m > 100
    np.testing.assert_array_equal(xr, x)
    np.testing.assert_array_equal(ar, a)
    np.testing.assert_array_equal(vr, v)


def test_merge_case_moves_chain_heads_far():
    """Most chain heads absorb all five followers, the last one 1.0 r from
    the head's start: four times the reach (0.25 (r_i + r_j)) of a pair test
    made at entry, so these merges need the direct scan of pgpu_merge."""
    w, n_elig, _ = cases.merge_clusters(seed=0, chains=10)
    _, ar, vr, _ = O.restate_merge(w, n_elig)
    full = sum(bool(np.all(ar[6 * c + 1:6 * c + 6] == 0.0) and np.all(vr[6 * c + 1:6 * c + 6] == 0.0))
               for c in range(10))
    assert full >= 8


def test_restated_merge_conserves_total_strength():
    w, n_elig, _ = cases.merge_clusters(seed=1)
    _, ar, _, m = O.restate_merge(w, n_elig)
    assert m > 0
    np.testing.assert_allclose(ar.sum(0), w.alpha.sum(0), rtol=0, atol=1e-15)


# ---------------------------------------------------------------- GPU

def gpu_merge(w, n_elig, precision=capi.FP64):
    with capi.Context(precision=precision, nu=1e-4) as c:
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        m = c.merge(k, n_elig)
        x, a, s, v = c.particles(k)
    return x, a, s, v, m


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32C])
def test_gpu_merge_matches_pawan(gpu, ref_available, seed, prec):
    w, n_elig, active = cases.merge_clusters(seed=seed)
    x, a, _, v = pawan_merge(w, active)
    gx, ga, gs, gv, m = gpu_merge(w, n_elig, prec)
    np.testing.assert_array_equal(gx, x)
    np.testing.assert_array_equal(ga, a)
    np.testing.assert_array_equal(gv, v)
    np.testing.assert_array_equal(gs, w.sigma)
    assert m == O.restate_merge(w, n_elig)[3]


@pytest.mark.gpu
def test_gpu_merge_edge_cases(gpu):
    w, n_elig, _ = cases.merge_clusters(seed=3)
    # nothing eligible: nothing changes
    gx, ga, _, gv, m = gpu_merge(w, 0)
    assert m == 0
    np.testing.assert_array_equal(gx, w.pos)
    np.testing.assert_array_equal(ga, w.alpha)
    # more than n eligible: the whole wake
    gx, ga, _, gv, m = gpu_merge(w, 10 * w.n)
    xr, ar, vr, mr = O.restate_merge(w, w.n)
    assert m == mr
    np.testing.assert_array_equal(gx, xr)
    np.testing.assert_array_equal(ga, ar)
    # one particle; all strengths zero
    one = w.subset(1)
    assert gpu_merge(one, 1)[4] == 0
    zero = cases.Wake(w.pos, np.zeros_like(w.alpha), w.sigma, w.vol)
    assert gpu_merge(zero, w.n)[4] == 0
    with capi.Context(precision=capi.FP64) as c:
        k = c.add_wake(4)
        c.set_particles(k, w.subset(4))
        with pytest.raises(capi.PgpuError, match="negative"):
            c.merge(k, -1)


@pytest.mark.gpu
def test_gpu_merge_dense_cluster_regrows_candidates(gpu):
    """800 particles inside one merge reach: 319600 candidate pairs, more than
    the first candidate buffer (65536) holds."""
    rng = np.random.default_rng(5)
    n = 800
    pos = rng.normal(scale=0.004, size=(n, 3))
    alpha = rng.normal(size=(n, 3)) * 1e-3
    w = cases.Wake(pos, alpha, np.full(n, 0.1), np.full(n, 1e-4))
    gx, ga, _, gv, m = gpu_merge(w, n)
    xr, ar, vr, mr = O.restate_merge(w, n)
    assert m == mr > 0
    np.testing.assert_array_equal(gx, xr)
    np.testing.assert_array_equal(ga, ar)
    np.testing.assert_array_equal(gv, vr)


@pytest.mark.gpu
def test_gpu_merge_200k_jittered_ring_vs_restatement(gpu):
    """200k particles (ring, Gaussian cross-section, sigma 0.02) with every
    strength turned 0.02 rad about a random axis: ~6e4 merges."""
    w = cases.jittered(cases.ring_gaussian(stations=200, per_section=1000), 0.02, seed=1)
    gx, ga, _, gv, m = gpu_merge(w, w.n, capi.FP32C)
    xr, ar, vr, mr = O.restate_merge(w, w.n)
    print(f"200k jittered ring: {m} merges")
    assert m == mr > 10000
    np.testing.assert_array_equal(gx, xr)
    np.testing.assert_array_equal(ga, ar)
    np.testing.assert_array_equal(gv, vr)


@pytest.mark.gpu
def test_gpu_merge_one_wake_of_two_systems_then_solve(gpu):
    """The merge touches only its wake (here the second of the device
    layout), and the next solve sees the merged particles: rates equal those
    of a fresh context of the same layout given the merged wake."""
    w, n_elig, _ = cases.merge_clusters(seed=4)
    other = cases.ring_stations(stations=20, seed=9)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        e = c.add_wake(other.n, 0)
        k = c.add_wake(w.n, 1)
        c.set_particles(e, other)
        c.set_particles(k, w)
        m = c.merge(k, n_elig)
        x, a, s, v = c.particles(k)
        ox, oa, _, _ = c.particles(e)
        c.solve()
        vel, dal = c.rates(k)
    xr, ar, vr, mr = O.restate_merge(w, n_elig)
    assert m == mr
    np.testing.assert_array_equal(x, xr)
    np.testing.assert_array_equal(ox, other.pos)
    np.testing.assert_array_equal(oa, other.alpha)
    merged = cases.Wake(x, a, s, v)
    with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
        e = c.add_wake(other.n, 0)
        k = c.add_wake(w.n, 1)
        c.set_particles(e, other)
        c.set_particles(k, merged)
        c.solve()
        vel2, dal2 = c.rates(k)
    np.testing.assert_array_equal(vel, vel2)
    np.testing.assert_array_equal(dal, dal2)
