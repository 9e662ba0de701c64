"""Conservation drift and the FP32C trajectory against the FP64 one.

    python -m pawan_b200.conservation [--stations 200] [--steps 50] [--every 10] [--json out.json]

Advances the Gaussian-core vortex ring of the 1M benchmark geometry
(``stations`` x 1000 particles, R = 1, a = 0.1, sigma = 0.02, seed 1,
nu = 1e-4) with RK4, dt = 0.005, on the GPU in both precision modes from the
same initial state.  Every ``every`` steps it records, per mode, the
diagnostics of pgpu_diagnose (interaction.cpp:64-194) and reports:

* drift of each conserved or slowly varying quantity, |Q(t) - Q(0)| / S,
  with S a scale of the same units that does not vanish for a ring:
  total vorticity, S = sum_i |alpha_i| (a closed ring has Q(0) = 0); linear
  impulse, S = |Q(0)|; angular impulse, S = sum_i |alpha_i| |x_i|^2 (Q(0) = 0
  for a ring); helicity, S = the kinetic energy at step 0 (same units, and
  Q(0) = 0 without swirl); kinetic energies, S = their value at step 0 (they
  decay with viscosity);
* the FP32C trajectory against the FP64 one: max-norm relative difference of
  the displacement x(t) - x(0) and of the strengths alpha(t).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import capi, cases

NAMES = ["total vorticity", "linear impulse", "angular impulse", "helicity", "kinetic energy", "kinetic energy F"]


def quantities(d: np.ndarray) -> dict[str, np.ndarray]:
    """Split the 15-value diagnostic record into named quantities."""
    return {"total vorticity": d[0:3], "linear impulse": d[3:6], "angular impulse": d[6:9],
            "helicity": d[9:10], "kinetic energy": d[12:13], "kinetic energy F": d[13:14]}


def rel_diff(x: np.ndarray, ref: np.ndarray) -> float:
    """Max-norm relative difference, max_i |x_i - ref_i| / max_i |ref_i| (row norms for (n, 3))."""
    num = np.linalg.norm(x - ref, axis=-1).max() if x.ndim > 1 else np.abs(x - ref).max()
    den = np.linalg.norm(ref, axis=-1).max() if ref.ndim > 1 else np.abs(ref).max()
    return float(num / den) if den > 0 else float(num)


def run(stations: int = 200, steps: int = 50, every: int = 10, dt: float = 0.005, nu: float = 1e-4) -> dict:
    w = cases.ring_gaussian(stations=stations, per_section=1000, sigma=0.02, seed=1)
    amag = float(np.linalg.norm(w.alpha, axis=1).sum())
    scale_a = float((np.linalg.norm(w.alpha, axis=1) * (w.pos ** 2).sum(axis=1)).sum())
    ctx = {}
    for name, prec in (("fp32c", capi.FP32C), ("fp64", capi.FP64)):
        c = capi.Context(precision=prec, nu=nu)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        ctx[name] = (c, k)
    records = []
    q0 = {}
    t = 0
    while True:
        rec = {"step": t}
        states = {}
        for name, (c, k) in ctx.items():
            d, _ = c.diagnose(0)
            q = quantities(d)
            if t == 0:
                q0[name] = q
            scale = {"total vorticity": amag, "linear impulse": float(np.linalg.norm(q0[name]["linear impulse"])),
                     "angular impulse": scale_a, "helicity": float(abs(q0[name]["kinetic energy"][0])),
                     "kinetic energy": float(abs(q0[name]["kinetic energy"][0])),
                     "kinetic energy F": float(abs(q0[name]["kinetic energy F"][0]))}
            rec[name] = {qn: float(np.linalg.norm(q[qn] - q0[name][qn]) / scale[qn]) for qn in NAMES}
            rec[name + "_values"] = {qn: q[qn].tolist() for qn in NAMES}
            states[name] = c.state(k)
        rec["fp32c_vs_fp64"] = {"displacement": rel_diff(states["fp32c"][0] - w.pos, states["fp64"][0] - w.pos)
                                if t else 0.0,
                                "alpha": rel_diff(states["fp32c"][1], states["fp64"][1])}
        records.append(rec)
        if t >= steps:
            break
        n = min(every, steps - t)
        for c, _ in ctx.values():
            c.step("rk4", dt, n)
        for c, _ in ctx.values():
            c.sync()
        t += n
    for c, _ in ctx.values():
        c.close()
    return {"particles": w.n, "steps": steps, "dt": dt, "nu": nu, "records": records}


def markdown(res: dict) -> str:
    lines = [f"N = {res['particles']}, RK4 dt = {res['dt']}, nu = {res['nu']}", "",
             "| step | mode | " + " | ".join(NAMES) + " |", "|---|---|" + "---|" * len(NAMES)]
    for r in res["records"]:
        for mode in ("fp32c", "fp64"):
            lines.append(f"| {r['step']} | {mode} | " + " | ".join(f"{r[mode][q]:.2e}" for q in NAMES) + " |")
    lines += ["", "| step | FP32C vs FP64: displacement | alpha |", "|---|---|---|"]
    for r in res["records"]:
        lines.append(f"| {r['step']} | {r['fp32c_vs_fp64']['displacement']:.2e} | {r['fp32c_vs_fp64']['alpha']:.2e} |")
    return "\n".join(lines)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--stations", type=int, default=200)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    res = run(a.stations, a.steps, a.every, a.dt)
    print(markdown(res))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
