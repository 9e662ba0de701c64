"""The oracle itself: PAWAN's own compiled code vs the golden fixtures it
produced, and the FP64 restatement vs PAWAN's own code (CPU only)."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import cases

GOLD = Path(__file__).resolve().parent / "golden"


def _digest(w):
    h = hashlib.sha256()
    for a in (w.pos, w.alpha, w.sigma, w.vol):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def test_generators_reproduce_fixture_inputs():
    g = np.load(GOLD / "ring1000.npz")
    w = cases.ring_stations(stations=40, seed=0)
    assert _digest(w) == str(g["sha256"])
    np.testing.assert_array_equal(w.pos, g["pos"])
    g5 = np.load(GOLD / "ring5000.npz")
    assert _digest(cases.ring_stations()) == str(g5["sha256"])


def test_ring5000_layout():
    w = cases.ring_stations()
    assert w.n == 5000
    # total strength of one station = Gamma R dpsi along the tangent
    st = w.alpha.reshape(200, 25, 3).sum(1)
    np.testing.assert_allclose(np.linalg.norm(st, axis=1), 2 * np.pi / 200, rtol=1e-12)


def test_reference_reproduces_golden(ref_available):
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    R = O.RefSystem([w], float(g["nu"]))
    R.solve()
    v, a = R.rates()
    # PAWAN's OpenMP reductions combine thread partials in arrival order, so
    # reruns agree to rounding, not bit for bit.
    assert O.rel_err(v, g["vel"]) < 1e-14
    assert O.rel_err(a, g["dalpha"]) < 1e-14
    np.testing.assert_allclose(R.diagnose()[3:], g["diag"][3:], rtol=1e-12, atol=1e-15)


def test_restatement_rates_vs_golden():
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    v, a = O.restate_rates(w, float(g["nu"]))
    assert O.rel_err(v, g["vel"]) < 1e-12
    assert O.rel_err(a, g["dalpha"]) < 1e-12


def test_restatement_rates_sampled_5000():
    g = np.load(GOLD / "ring5000.npz")
    w = cases.ring_stations()
    v, a = O.restate_rates(w, float(g["nu"]), targets=g["rows"])
    assert O.rel_err(v, g["vel"]) < 1e-12
    assert O.rel_err(a, g["dalpha"]) < 1e-12


@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_restatement_steps_vs_golden(scheme):
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    x, al = O.restate_step(w, float(g["nu"]), scheme, float(g["dt"]), 2)
    assert O.rel_err(x, g[f"{scheme}_pos"]) < 1e-13
    assert O.rel_err(al, g[f"{scheme}_alpha"]) < 1e-12


def test_restatement_diagnostics_vs_golden():
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    d, vbi = O.restate_diagnose(w)
    ref = g["diag"]
    scale = np.maximum(np.abs(ref), 1e-12 * np.abs(ref).max())
    # total vorticity is a cancelling sum of O(1e-2) terms: compare absolutely
    assert np.all(np.abs(d[:3] - ref[:3]) < 1e-14)
    assert np.all(np.abs(d[3:] - ref[3:]) <= 1e-11 * scale[3:] + 1e-15)
    np.testing.assert_allclose(vbi, g["vbi"], rtol=1e-12, atol=1e-15)


def test_restatement_two_wakes_vs_golden():
    g = np.load(GOLD / "twowake.npz")
    w1 = cases.Wake(g["pos1"], g["alpha1"], g["sigma1"], g["vol1"])
    w2 = cases.Wake(g["pos2"], g["alpha2"], g["sigma2"], g["vol2"])
    wc = cases.Wake.concat([w1, w2])
    v, a = O.restate_rates(wc, float(g["nu"]))
    assert O.rel_err(v, np.concatenate([g["vel1"], g["vel2"]])) < 1e-12
    assert O.rel_err(a, np.concatenate([g["dalpha1"], g["dalpha2"]])) < 1e-12
    d, _ = O.restate_diagnose(wc, [0, w1.n, wc.n])
    np.testing.assert_allclose(d[3:], g["diag"][3:], rtol=1e-11, atol=1e-14)


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's input (one strength flipped) must be
    visible at the 1e-5 gate the GPU FP32 path is held to."""
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"].copy(), g["sigma"], g["vol"])
    w.alpha[17] *= -1.0
    v, a = O.restate_rates(w, float(g["nu"]))
    assert O.rel_err(v, g["vel"]) > 1e-5 or O.rel_err(a, g["dalpha"]) > 1e-5


def test_reference_integrate_files_present():
    d = GOLD / "integrate"
    wake = (d / "ring1000_rk4.wake").read_bytes()
    diag = (d / "ring1000_rk4.diagnosis").read_bytes()
    # .wake: per record t, nWake, maxN (written with sizeof(size_t)), then the wake
    n = 1000
    rec = 8 + 8 + 8 + 8 + n * (3 + 3 + 1 + 1 + 1 + 1) * 8
    assert len(wake) == 4 * rec
    # .diagnosis: nu, then per record t + 15 doubles
    assert len(diag) == 8 + 4 * 16 * 8


def test_restated_vorticity_field_matches_pawan_influence(ref_available):
    """The FP64 restatement of influence() against PAWAN's own resolve() on two
    interacting wakes (interaction.cpp:212-260)."""
    w1 = cases.ring_stations(stations=40, seed=0)
    w2 = cases.ring_stations(stations=30, R=0.7, seed=1)
    with O.quiet():
        R = O.RefSystem([w1, w2], 1e-4)
        k = R.vorticity_field()
        R.close()
    kr = O.restate_vorticity_field(cases.Wake.concat([w1, w2]))
    assert O.rel_err(kr, k) < 1e-13
