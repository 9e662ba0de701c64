"""A small, self-contained workload for profilers (ncu) and quick timing.

    python -m pawan_b200.profile_case [--stations 200] [--solves 3] [--fp64] [--steps 1] [--block 256 --tpt 2]

Builds the Gaussian-core vortex ring of the 1M-particle benchmark with
``stations`` x 1000 particles (200 -> N = 200,000), runs ``solves`` rate
evaluations, ``steps`` RK4 steps and one diagnose on cuda:0 through the C ABI,
and prints the pair-kernel time per launch.  Sized so that an ncu capture of
one pair-kernel launch ends in about a minute.
"""
from __future__ import annotations

import argparse

from . import capi, cases


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--stations", type=int, default=200)
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--block", type=int, default=0, help="pair-kernel block size (0: library default)")
    ap.add_argument("--tpt", type=int, default=0, help="targets per thread (0: library default)")
    ap.add_argument("--sigma", type=float, default=0.02, help="smoothing radius (smaller: fewer near pairs)")
    a = ap.parse_args()
    w = cases.ring_gaussian(stations=a.stations, per_section=1000, sigma=a.sigma, seed=1)
    c = capi.Context(precision=capi.FP64 if a.fp64 else capi.FP32C, nu=1e-4, block=a.block, tpt=a.tpt)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    for _ in range(a.solves):
        c.solve()
    c.sync()
    ms, nl = c.pair_kernel_time()
    pairs, full = c.pair_counts()
    print(f"N {w.n} pair kernel {ms / max(nl, 1):.3f} ms/launch, {w.n * (w.n - 1) / (ms / max(nl, 1) / 1e3):.3e} pairs/s, "
          f"full-formula fraction {full / max(pairs, 1):.4f}")
    if a.steps:
        c.step("rk4", 0.005, a.steps)
        c.sync()
    d, vbi = c.diagnose(0)
    print("diagnostics", d.tolist(), "vbi", vbi.tolist())
    c.close()


if __name__ == "__main__":
    main()
