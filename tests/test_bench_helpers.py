"""Host-side arithmetic of bench.py (no GPU): the roofline under both flop
conventions, the pair-count extrapolation of the CPU samples, the seeded
sample, and the reference arm's JSON line on a small ring."""
import json
import math
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_pair_roofline_conventions():
    # two launches of 1e12 ordered pairs, 3% full-formula, 1.0 s each
    pairs, full = 2 * 10**12, 6 * 10**10
    r = bench.pair_roofline(2000.0, 2, pairs, full, peak=70.0)
    counted = (95 * full + 59 * (pairs - full)) / 2 / 1.0 / 1e12
    assert math.isclose(r["achieved"], counted, rel_tol=1e-12)
    assert math.isclose(r["achieved_flat95"], 95 * pairs / 2 / 1e12, rel_tol=1e-12)
    assert math.isclose(r["frac"], counted / 70.0, rel_tol=1e-12)
    assert math.isclose(r["full_pair_fraction"], 0.03, rel_tol=1e-12)
    assert r["pair_kernel_ms"] == 1000.0
    # a kernel that evaluated only far pairs is rated at 59 flop per pair
    assert math.isclose(bench.pair_roofline(1000.0, 1, 10**12, 0, 1.0)["achieved"], 59.0, rel_tol=1e-12)


def test_extrapolation_by_pair_count():
    # a 6000-particle step of 3 s extrapolates to N = 1M by N(N-1) / (n(n-1))
    sps = bench.extrapolate_steps_per_s(3.0, 6000, 1_000_000)
    assert math.isclose(1.0 / sps, 3.0 * (1e6 * (1e6 - 1)) / (6000 * 5999), rel_tol=1e-12)
    assert math.isclose(bench.extrapolate_steps_per_s(2.0, 100, 100), 0.5, rel_tol=1e-12)


def test_sample_is_seeded_and_ordered():
    w = bench.workload(4)
    a, b = bench.sample(w, 500), bench.sample(w, 500)
    np.testing.assert_array_equal(a.pos, b.pos)
    np.testing.assert_array_equal(a.alpha, b.alpha)
    assert a.n == 500
    # rows keep the ring's order (a sorted subset), so each row is one of the ring's particles
    rows = [np.flatnonzero((w.pos == p).all(axis=1))[0] for p in a.pos[:20]]
    assert rows == sorted(rows)


def test_reference_arm_line(ref_available):
    """bench.py --impl reference on a 10,000-particle ring: one JSON line with
    the contract's keys, its e2e equal to its value, and the CPU baseline
    describing the run."""
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--stations", "10"], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["metric"] == "RK4 steps/s" and line["unit"] == "steps/s"
    assert line["config"]["particles"] == 10_000 and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1
    assert math.isclose(line["ms_per_step"], 1e3 / line["value"], rel_tol=1e-9)
