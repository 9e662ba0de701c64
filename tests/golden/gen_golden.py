"""Generates the golden fixtures under tests/golden/ from PAWAN's own code.

    make -C oracle && python tests/golden/gen_golden.py [name ...]

Every output comes from ``oracle/_ref/libpawanref.so``: PAWAN's unmodified
interaction / parallel / integration / wake sources compiled against the
project's GSL-subset shim (``oracle/Makefile``); the ``*_ho`` fixtures come
from ``oracle/_ref/libpawanref_ho.so``, the same sources built with PAWAN's
high-order algebraic kernel (src/interaction/highorder.h).  Inputs come from the seeded
generators in ``pawan_b200.cases``; their SHA-256 is stored so a test can
check that regenerating the inputs reproduces the fixture's inputs.

Fixtures:
  ring1000.npz   - 40-station ring (N=1000, sigma=0.1, nu=1e-4): inputs, rates
                   of one solve, diagnostics and vbi, state after 2 RK4 steps
                   and after 2 RK3 steps (dt=0.01).
  ring5000.npz   - the 5000-particle ring (200 stations x 25, seed 0): rates on
                   256 sampled rows, diagnostics, and the sampled rows of the
                   state after one RK4 step (dt=0.01).
  twowake.npz    - two interacting wakes in one system (leapfrog pair, N=400+320).
  integrate/     - the .wake / .diagnosis files of PAWAN's own
                   __integration::integrate for 3 RK4 steps of ring1000.
  ring1000_ho.npz - ring1000's inputs (checked by SHA-256) with the high-order
                   kernel: rates, diagnostics (enstrophy and enstrophyF are
                   non-zero for it) and vbi, the vorticity field of
                   influence(), the state after 2 RK4 and after 2 RK3 steps.
  twowake_ho.npz - twowake's inputs with the high-order kernel: rates of both
                   wakes and the diagnostics (cross-wake enstrophy terms).
  ring5000_long.npz - the 5000-particle ring advanced by PAWAN's own __rk4
                   (dt=0.01, nu=1e-4) for 100 steps: diagnostics at steps 0,
                   1, 10 and 100, and the state of 256 sampled rows at steps 1,
                   10 and 100 (about 10 minutes on 8 host cores).
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from pawan_b200 import cases  # noqa: E402

OUT = Path(__file__).resolve().parent
NU = 1e-4


def digest(w) -> str:
    h = hashlib.sha256()
    for a in (w.pos, w.alpha, w.sigma, w.vol):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def ring1000():
    w = cases.ring_stations(stations=40, seed=0)
    R = O.RefSystem([w], NU)
    R.solve()
    vel, da = R.rates()
    diag = R.diagnose()
    vbi = R.getvi([0.0, 0.0, 0.0])
    R.step("rk4", 0.01, 2)
    x4, a4 = R.state()
    R3 = O.RefSystem([w], NU)
    R3.step("rk3", 0.01, 2)
    x3, a3 = R3.state()
    np.savez_compressed(OUT / "ring1000.npz", pos=w.pos, alpha=w.alpha, sigma=w.sigma, vol=w.vol, nu=NU,
                        vel=vel, dalpha=da, diag=diag, vbi=vbi, rk4_pos=x4, rk4_alpha=a4, rk3_pos=x3,
                        rk3_alpha=a3, dt=0.01, sha256=digest(w))


def ring5000():
    w = cases.ring_stations()
    rows = np.sort(np.random.default_rng(123).choice(w.n, 256, replace=False))
    R = O.RefSystem([w], NU)
    R.solve()
    vel, da = R.rates()
    diag = R.diagnose()
    vbi = R.getvi([0.0, 0.0, 0.0])
    R.step("rk4", 0.01, 1)
    x4, a4 = R.state()
    np.savez_compressed(OUT / "ring5000.npz", rows=rows, vel=vel[rows], dalpha=da[rows], diag=diag, vbi=vbi,
                        rk4_pos=x4[rows], rk4_alpha=a4[rows], dt=0.01, nu=NU, sha256=digest(w))


def twowake():
    w1 = cases.ring_stations(stations=16, seed=3)
    w2 = cases.ring_stations(R=1.2, stations=16, z0=0.3, seed=5).subset(320)
    R = O.RefSystem([w1, w2], NU)
    R.solve()
    v1, d1 = R.rates(0)
    v2, d2 = R.rates(1)
    diag = R.diagnose()
    np.savez_compressed(OUT / "twowake.npz", pos1=w1.pos, alpha1=w1.alpha, sigma1=w1.sigma, vol1=w1.vol,
                        pos2=w2.pos, alpha2=w2.alpha, sigma2=w2.sigma, vol2=w2.vol, vel1=v1, dalpha1=d1,
                        vel2=v2, dalpha2=d2, diag=diag, nu=NU)


def ring1000_ho():
    w = cases.ring_stations(stations=40, seed=0)
    R = O.RefSystem([w], NU, kernel="highorder")
    R.solve()
    vel, da = R.rates()
    diag = R.diagnose()
    vbi = R.getvi([0.0, 0.0, 0.0])
    field = R.vorticity_field()
    R.step("rk4", 0.01, 2)
    x4, a4 = R.state()
    R3 = O.RefSystem([w], NU, kernel="highorder")
    R3.step("rk3", 0.01, 2)
    x3, a3 = R3.state()
    np.savez_compressed(OUT / "ring1000_ho.npz", nu=NU, vel=vel, dalpha=da, diag=diag, vbi=vbi, field=field,
                        rk4_pos=x4, rk4_alpha=a4, rk3_pos=x3, rk3_alpha=a3, dt=0.01, sha256=digest(w))


def twowake_ho():
    w1 = cases.ring_stations(stations=16, seed=3)
    w2 = cases.ring_stations(R=1.2, stations=16, z0=0.3, seed=5).subset(320)
    R = O.RefSystem([w1, w2], NU, kernel="highorder")
    R.solve()
    v1, d1 = R.rates(0)
    v2, d2 = R.rates(1)
    diag = R.diagnose()
    np.savez_compressed(OUT / "twowake_ho.npz", vel1=v1, dalpha1=d1, vel2=v2, dalpha2=d2, diag=diag, nu=NU,
                        sha256=digest(w1) + digest(w2))


def ring5000_long():
    w = cases.ring_stations()
    rows = np.sort(np.random.default_rng(321).choice(w.n, 256, replace=False))
    R = O.RefSystem([w], NU)
    out = {"rows": rows, "dt": 0.01, "nu": NU, "sha256": digest(w), "steps": np.array([0, 1, 10, 100])}
    out["diag0"] = R.diagnose()
    done = 0
    for k in (1, 10, 100):
        R.step("rk4", 0.01, k - done)
        done = k
        x, a = R.state()
        out[f"pos{k}"], out[f"alpha{k}"] = x[rows], a[rows]
        out[f"diag{k}"] = R.diagnose()
    np.savez_compressed(OUT / "ring5000_long.npz", **out)


def integrate_files():
    d = OUT / "integrate"
    d.mkdir(exist_ok=True)
    w = cases.ring_stations(stations=40, seed=0)
    R = O.RefSystem([w], NU)
    R.integrate("rk4", 0.03, 3, True, str(d / "ring1000_rk4"))


FIXTURES = {"ring1000": ring1000, "ring5000": ring5000, "twowake": twowake, "integrate": integrate_files,
            "ring1000_ho": ring1000_ho, "twowake_ho": twowake_ho, "ring5000_long": ring5000_long}

if __name__ == "__main__":
    for name in sys.argv[1:] or FIXTURES:
        FIXTURES[name]()
    for p in sorted(OUT.rglob("*")):
        if p.is_file() and p.suffix != ".py":
            print(p.relative_to(OUT), p.stat().st_size)
