"""Long-horizon parity of the 5000-particle ring, and the batched uneven rings
with the per-size-class autotuner.

* The 5000-particle ring (200 stations x 25, sigma = 0.1, seed 0, nu = 1e-4,
  RK4 dt = 0.01) stepped 100 times on the GPU against PAWAN's own __rk4 run
  (tests/golden/ring5000_long.npz): 256 sampled rows of the state at steps 1,
  10 and 100, and the diagnostics there.  Gates: FP64 1e-10, FP32C 1e-5.
* pgpu_autotune_classes: the cache file round trip, the per-class launch
  (one pair launch per distinct class shape) against the single launch, and
  100 RK4 steps of the 8 smallest of the 64 uneven rings in one batched
  context against the FP64 restatement of each of the 3 smallest alone.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

GOLD = Path(__file__).resolve().parent / "golden"
TOL = {capi.FP64: 1e-10, capi.FP32C: 1e-5}
PREC = [capi.FP64, capi.FP32C]


def load_long():
    return np.load(GOLD / "ring5000_long.npz")


def test_long_fixture_inputs_match_generator():
    """The fixture was made from the seeded generator's 5000-particle ring."""
    import hashlib
    g = load_long()
    w = cases.ring_stations()
    h = hashlib.sha256()
    for a in (w.pos, w.alpha, w.sigma, w.vol):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    assert str(g["sha256"]) == h.hexdigest()
    assert list(g["steps"]) == [0, 1, 10, 100]


def diag_err(d, ref, scale):
    """Per-quantity |d - ref| / max(|ref|, scale) over the 15 diagnostics,
    with `scale` the ring's kinetic energy for the quantities that vanish."""
    return np.abs(d - ref) / np.maximum(np.abs(ref), scale)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PREC)
def test_ring5000_100_rk4_steps_vs_pawan(gpu, prec):
    g = load_long()
    w = cases.ring_stations()
    rows = g["rows"]
    c = capi.Context(precision=prec, nu=float(g["nu"]))
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    d0, _ = c.diagnose(0)
    scale = abs(float(g["diag0"][12]))  # kinetic energy
    assert np.all(diag_err(d0, g["diag0"], scale) < TOL[prec])
    done = 0
    worst = {}
    for step in (1, 10, 100):
        c.step("rk4", float(g["dt"]), step - done)
        done = step
        x, a = c.state(k)
        ex, ea = O.rel_err(x[rows], g[f"pos{step}"]), O.rel_err(a[rows], g[f"alpha{step}"])
        d, _ = c.diagnose(0)
        ed = float(diag_err(d, g[f"diag{step}"], scale).max())
        worst[step] = (ex, ea, ed)
        assert ex < TOL[prec] and ea < TOL[prec] and ed < TOL[prec], (step, ex, ea, ed)
    c.close()
    # the drift of the diagnostics over the run is the reference's drift
    ref_drift = np.abs(g["diag100"] - g["diag0"]) / np.maximum(np.abs(g["diag0"]), scale)
    print(f"ring5000, 100 RK4 steps ({'FP64' if prec == capi.FP64 else 'FP32C'}): errors (pos, alpha, diag) "
          f"{worst}; PAWAN's own drift of the diagnostics over the run: max {ref_drift.max():.2e}")


# ------------------------------------------------------------------ size classes
def uneven_subset(k: int = 8):
    ws = cases.uneven_rings(count=64, nmin=2e3, nmax=2e5, seed=2)
    order = np.argsort([w.n for w in ws])
    return [ws[i] for i in order[:k]]


def batched(ws, prec=capi.FP32C, **kw):
    c = capi.Context(precision=prec, nu=1e-4, **kw)
    ids = [c.add_wake(w.n, i) for i, w in enumerate(ws)]
    for i, w in zip(ids, ws):
        c.set_particles(i, w)
    return c, ids


def cache_line(gpu_name, prec, cls, best, nshapes):
    ms = [10.0] * nshapes
    ms[best] = 1.0
    b, t = capi.kernel_shapes()[best]
    return json.dumps({"gpu": gpu_name, "precision": prec, "kernel": "gaussian", "class": cls, "nmin": 0,
                       "nmax": 0, "block": b, "tpt": t, "ms": ms})


@pytest.mark.gpu
def test_autotune_classes_cache_round_trip(gpu, tmp_path):
    ws = cases.uneven_rings(count=12, nmin=2e3, nmax=6e4, seed=9)
    cache = tmp_path / "tune.jsonl"
    c, _ = batched(ws)
    first = c.autotune_classes(reps=1, cache=str(cache))
    c.close()
    classes = sorted({capi_class(w.n) for w in ws})
    assert [x["class"] for x in first["classes"]] == classes
    assert all(not x["from_cache"] for x in first["classes"])
    assert sum(x["systems"] for x in first["classes"]) == len(ws)
    lines = [json.loads(s) for s in cache.read_text().splitlines()]
    assert [d["class"] for d in lines] == classes
    for x in first["classes"]:
        # the class's shape is its fastest, and the single shape within 2% of
        # it unless the classes launch separately
        ms = x["ms"]
        assert ms[f"{x['block']}x{x['tpt']}"] == min(ms.values())
        if not first["per_class"]:
            assert ms[f"{x['single_block']}x{x['single_tpt']}"] <= 1.02 * min(ms.values()) + 1e-9
    c, _ = batched(ws)
    second = c.autotune_classes(reps=1, cache=str(cache))
    c.close()
    assert all(x["from_cache"] for x in second["classes"])
    assert [(x["block"], x["tpt"]) for x in second["classes"]] == [(x["block"], x["tpt"]) for x in first["classes"]]


@pytest.mark.gpu
def test_autotune_classes_unwritable_cache_keeps_the_work_plan(gpu, tmp_path):
    """A cache file that cannot be written is reported after the tuning has
    put its choice in place: the context's rates afterwards are those of an
    untuned context (the timing launches leave no plan or partials behind)."""
    ws = cases.uneven_rings(count=12, nmin=2e3, nmax=6e4, seed=9)
    assert len({capi_class(w.n) for w in ws}) >= 2
    c, ids = batched(ws)
    with pytest.raises(capi.PgpuError, match="cannot append to the autotune cache"):
        c.autotune_classes(reps=1, cache=str(tmp_path / "no_such_dir" / "tune.jsonl"))
    c.solve()
    ref, rids = batched(ws)
    ref.solve()
    for i, r in zip(ids, rids):
        v, a = c.rates(i)
        vr, ar = ref.rates(r)
        # other shapes and chunk counts only reorder the FP32 group sums
        assert O.rel_err(v, vr) < 2e-6 and O.rel_err(a, ar) < 2e-6
    c.close()
    ref.close()


def capi_class(n: int) -> int:
    k, hi = 0, 4096
    while n >= hi:
        k, hi = k + 1, hi * 4
    return k


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PREC)
def test_per_class_launches_equal_single_launch(gpu, tmp_path, prec):
    """A cache that gives the small and the large class different shapes forces
    one pair launch per class; two RK4 steps then agree with the single-shape
    launch to rounding (only the summation order differs)."""
    import torch
    ws = uneven_subset(3) + [cases.ring_stations(R=1.0, stations=2000, sigma=0.1, seed=1)]  # 3 x ~2e3 and 5e4
    assert len({capi_class(w.n) for w in ws}) == 2
    name = torch.cuda.get_device_properties(0).name
    nshapes = len(capi.kernel_shapes())
    pname = "fp64" if prec == capi.FP64 else "fp32c"
    cache = tmp_path / "forced.jsonl"
    cls = sorted({capi_class(w.n) for w in ws})
    cache.write_text(cache_line(name, pname, cls[0], 0, nshapes) + "\n" + cache_line(name, pname, cls[1], 3, nshapes)
                     + "\n")
    c1, ids1 = batched(ws, prec)
    tune = c1.autotune_classes(reps=1, cache=str(cache))
    assert tune["per_class"] and all(x["from_cache"] for x in tune["classes"])
    l0 = c1.launch_count()
    c1.step("rk4", 0.005, 2)
    c1.sync()
    # 2 steps x 4 stages x (2 pair launches + 1 stage launch, + the source-box
    # launch ahead of the FP32C pair kernels)
    assert c1.launch_count() - l0 == 2 * 4 * (3 + (prec == capi.FP32C))
    c2, ids2 = batched(ws, prec, block=256, tpt=1)
    c2.step("rk4", 0.005, 2)
    tol = 1e-13 if prec == capi.FP64 else 2e-6
    for i1, i2 in zip(ids1, ids2):
        x1, a1 = c1.state(i1)
        x2, a2 = c2.state(i2)
        assert O.rel_err(x1, x2) < tol and O.rel_err(a1, a2) < tol
    c1.close()
    c2.close()


@pytest.mark.gpu
def test_uneven_rings_100_steps_vs_restatement(gpu):
    """The 8 smallest of the 64 uneven rings as 8 systems of one context,
    shapes autotuned per size class, 100 RK4 steps (dt = 0.005) replayed from
    the CUDA graph; the 3 smallest against the FP64 restatement of each ring
    stepped alone."""
    ws = uneven_subset(8)
    c, ids = batched(ws)
    c.autotune_classes(reps=1)
    c.step("rk4", 0.005, 100)
    c.sync()
    worst = 0.0
    for i in range(3):
        x, a = c.state(ids[i])
        xr, ar = O.restate_step(ws[i], 1e-4, "rk4", 0.005, 100)
        worst = max(worst, O.rel_err(x, xr), O.rel_err(a, ar))
    c.close()
    print(f"8 smallest uneven rings ({[w.n for w in ws]}), 100 RK4 steps: worst error of the 3 smallest {worst:.2e}")
    assert worst < TOL[capi.FP32C]
