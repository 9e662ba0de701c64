"""The seeded workload generators of pawan_b200.cases used by the merge and
rotor-wake tests and timings (CPU only)."""
import math

import numpy as np

from pawan_b200 import cases


def test_jittered_turns_every_strength_by_theta():
    w = cases.ring_stations(stations=40, seed=0)
    j = cases.jittered(w, 0.02, seed=1)
    np.testing.assert_array_equal(j.pos, w.pos)
    np.testing.assert_allclose(np.linalg.norm(j.alpha, axis=1), np.linalg.norm(w.alpha, axis=1), rtol=1e-14)
    cos = (j.alpha * w.alpha).sum(1) / (np.linalg.norm(j.alpha, axis=1) * np.linalg.norm(w.alpha, axis=1))
    # a rotation by theta about a random axis turns a vector by at most theta
    assert np.all(cos >= math.cos(0.02) - 1e-12)
    assert np.any(cos < 1 - 1e-6)
    # PAWAN's merge needs 1 - cos >= 1e-4; a 0.02 rad turn gives up to 2e-4
    assert (1 - cos).max() > 1e-4


def test_rotor_shedder_omega_sets_dt_only():
    a = cases.RotorShedder(per_blade=10)
    b = cases.RotorShedder(per_blade=10, omega=10.0)
    assert math.isclose(a.dt, math.radians(10.0)) and math.isclose(b.dt, a.dt / 10)
    for _ in range(3):
        wa, wb = a.shed(), b.shed()
        np.testing.assert_array_equal(wa.pos, wb.pos)
        np.testing.assert_array_equal(wa.alpha, wb.alpha)
    assert wa.n == 4 * 10


def test_merge_clusters_layout():
    w, n_elig, active = cases.merge_clusters(seed=0, chains=10)
    assert n_elig == int(0.8 * w.n) and active.shape == (w.n,)
    # PAWAN's loop (wake.cpp:115) visits particles while stepnum - active > 45; at stepnum 100 exactly
    # the first n_elig qualify
    ok = 100 - active > 45
    assert np.all(ok[:n_elig]) and not ok[n_elig]
    # chains come first: each follower's strength is perpendicular to the sum of those before it
    for c in range(10):
        tot = w.alpha[6 * c].copy()
        for k in range(1, 6):
            a = w.alpha[6 * c + k]
            assert abs(np.dot(a, tot)) < 1e-12 * np.linalg.norm(a) * np.linalg.norm(tot)
            tot = tot + a
    # zero-strength particles are present
    assert np.sum(np.all(w.alpha == 0.0, axis=1)) == 20
