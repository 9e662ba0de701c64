"""The growing rotor wake at its full density: 4 tip vortices shedding
200 particles per blade per step (10 deg per step, angular speed 10, so
dt = pi/180), Gamma = 0.05, core 0.02, sigma = 0.03, inflow 0.05 applied after
each RK3 step as PAWAN's operator split (wake.cpp:564-577).  Twenty steps on
the GPU against the oracle's FP64 restatement stepping the same sequence
(RK3 of rk3.cpp:12-65, inflow shift, then the new particles appended).

The filaments are dense: neighbours along a tip vortex sit ~9e-4 apart at
coordinates ~1, a few hundred FP32 ulps.  Rounding the positions to FP32 then
dominates the FP32C error; split positions (FP32 value + FP32 residual,
pgpu_config.split_positions) restore FP64-quality differences for near pairs.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import capi, cases

STEPS = 20
NU = 1e-4


@pytest.fixture(scope="module")
def reference():
    """FP64 restatement of the 20-step growing wake: per step the state, and
    the final state with its rates."""
    sh = cases.RotorShedder(per_blade=200, omega=10.0)
    w = sh.shed()
    vinf = np.asarray(sh.inflow)
    for _ in range(STEPS):
        x, a = O.restate_step(w, NU, "rk3", sh.dt, 1)
        w = cases.Wake(x + vinf * sh.dt, a, w.sigma, w.vol)
        w = cases.Wake.concat([w, sh.shed()])
    return w


def run_gpu(prec, split):
    sh = cases.RotorShedder(per_blade=200, omega=10.0)
    c = capi.Context(precision=prec, nu=NU, vinf=sh.inflow, split_positions=split)
    k = c.add_wake(4 * 200 * (STEPS + 1))
    c.set_particles(k, sh.shed())
    for _ in range(STEPS):
        c.step("rk3", sh.dt, 1)
        c.append_particles(k, sh.shed())
    c.sync()
    x, a = c.state(k)
    c.solve()
    v, da = c.rates(k)
    c.close()
    return x, a, v, da


@pytest.mark.gpu
@pytest.mark.parametrize("prec,split", [(capi.FP64, False), (capi.FP32C, False), (capi.FP32C, True)])
def test_rotor_wake_at_full_density(gpu, reference, prec, split):
    x, a, v, da = run_gpu(prec, split)
    w = reference
    assert x.shape[0] == w.n == 4 * 200 * (STEPS + 1)
    # trajectory: positions and strengths after 20 steps
    ex = O.rel_err(x, w.pos)
    ea = O.rel_err(a, w.alpha)
    # evaluation error at the GPU's own final state
    vr, dr = O.restate_rates(cases.Wake(x, a, w.sigma, w.vol), NU)
    evv, evd = O.rel_err(v, vr), O.rel_err(da, dr)
    tol = 1e-10 if prec == capi.FP64 else 1e-5
    print(f"rotor 200/blade, {STEPS} RK3 steps, {'FP64' if prec == capi.FP64 else 'FP32C'}"
          f"{' split' if split else ''}: state pos {ex:.2e} alpha {ea:.2e}; rates vel {evv:.2e} dalpha {evd:.2e}")
    assert ex < tol and ea < tol and evv < tol and evd < tol
    if split:
        # split positions remove the position rounding from the velocity (6e-6
        # without them); dalpha/dt keeps the FP32 rounding of the stretching
        # sums of nearly parallel strengths along the filament (~4e-6 either way)
        assert evv < 1e-6 and evd < 5e-6, (evv, evd)
