"""A small, self-contained workload for profilers (ncu) and quick timing.

    python -m pawan_b200.profile_case [--stations 200] [--solves 3] [--fp64] [--steps 1] [--block 256 --tpt 2]
    python -m pawan_b200.profile_case --surrogate 200000 [--solves 2]
    python -m pawan_b200.profile_case --mlp-train 20
    python -m pawan_b200.profile_case --kernel highorder [--stations 200]
    python -m pawan_b200.profile_case --merge [--stations 200]
    python -m pawan_b200.profile_case --workload ring5k|uneven64|rotor [--steps K]

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
    ap.add_argument("--surrogate", type=int, default=0,
                    help="instead: octree far field (order 2) on two coaxial rings of this many particles")
    ap.add_argument("--mlp-train", type=int, default=0,
                    help="instead: this many training steps of the far-field network (batch 65536)")
    ap.add_argument("--kernel", choices=sorted(capi.KERNELS), default="gaussian", help="regularisation kernel")
    ap.add_argument("--merge", action="store_true",
                    help="instead: one particle merge (pgpu_merge) of the ring with strengths turned 0.02 rad")
    ap.add_argument("--workload", choices=["ring5k", "uneven64", "rotor"], default=None,
                    help="instead: time steps of another ring workload (see workload_case)")
    ap.add_argument("--omega", type=float, default=1.0, help="rotor angular speed of --workload rotor (dt = 10 deg / omega)")
    a = ap.parse_args()
    if a.workload:
        workload_case(a.workload, a.steps, a.omega)
        return
    if a.merge:
        merge_case(a.stations)
        return
    if a.surrogate:
        surrogate_case(a.surrogate, a.solves)
        return
    if a.mlp_train:
        mlp_case(a.mlp_train)
        return
    w = cases.ring_gaussian(stations=a.stations, per_section=1000, sigma=a.sigma, seed=1)
    c = capi.Context(precision=capi.FP64 if a.fp64 else capi.FP32C, nu=1e-4, block=a.block, tpt=a.tpt,
                     kernel=a.kernel)
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
    import time
    c.sync()
    t = time.perf_counter()
    d, vbi = c.diagnose(0)
    print(f"diagnose {1e3 * (time.perf_counter() - t):.1f} ms; diagnostics", d.tolist(), "vbi", vbi.tolist())
    c.close()


def workload_case(name: str, steps: int, omega: float = 1.0) -> None:
    """Device time of whole steps, after the first (graph capture) step:

    ring5k    the 5000-particle ring (200 stations x 25, sigma 0.1, seed 0),
              RK4 dt = 0.01, FP64 and FP32C;
    uneven64  64 independent rings with N log-uniform in [2e3, 2e5] (seed 2)
              as 64 systems of one context, RK4 dt = 0.005, FP32C, autotuned;
    rotor     the growing 4-blade tip-vortex wake (200 particles per blade per
              step, 10 deg per step at angular speed omega, RK3, inflow 0.05
              after each step, FP32C) from its first segment for `steps`
              steps; reports the time per step at the end, the pair count so
              far and the largest strength (a bounded run keeps it near the
              shed strength).
    """
    import time
    steps = max(steps, 1)
    if name == "ring5k":
        w = cases.ring_stations(seed=0)
        for prec in (capi.FP64, capi.FP32C):
            with capi.Context(precision=prec, nu=1e-4) as c:
                k = c.add_wake(w.n)
                c.set_particles(k, w)
                c.step("rk4", 0.01, 1)
                c.sync()
                t = time.perf_counter()
                c.step("rk4", 0.01, steps)
                c.sync()
                dt = (time.perf_counter() - t) / steps
            print(f"ring5k {'FP64' if prec == capi.FP64 else 'FP32C'}: {1e3 * dt:.3f} ms per RK4 step, "
                  f"{1 / dt:.1f} steps/s, {4 * w.n * (w.n - 1) / dt:.3e} pairs/s")
    elif name == "uneven64":
        ws = cases.uneven_rings(count=64, nmin=2e3, nmax=2e5, seed=2)
        with capi.Context(precision=capi.FP32C, nu=1e-4) as c:
            ids = [c.add_wake(w.n, i) for i, w in enumerate(ws)]
            for i, w in zip(ids, ws):
                c.set_particles(i, w)
            c.autotune()
            c.step("rk4", 0.005, 1)
            c.sync()
            t = time.perf_counter()
            c.step("rk4", 0.005, steps)
            c.sync()
            dt = (time.perf_counter() - t) / steps
        n = sum(w.n for w in ws)
        pairs = sum(w.n * (w.n - 1) for w in ws)
        print(f"uneven64: {n} particles in 64 systems, {1e3 * dt:.1f} ms per RK4 step, {4 * pairs / dt:.3e} pairs/s")
    else:
        sh = cases.RotorShedder(omega=omega)
        cap = 4 * sh.per_blade * (steps + 1)
        with capi.Context(precision=capi.FP32C, nu=1e-4, vinf=sh.inflow) as c:
            k = c.add_wake(cap)
            c.set_particles(k, sh.shed())
            pairs = 0
            t0 = time.perf_counter()
            t_last = t0
            for it in range(steps):
                n = c.num_particles(k)
                pairs += 3 * n * (n - 1)
                if it == steps - 1:
                    c.sync()
                    t_last = time.perf_counter()
                c.step("rk3", sh.dt, 1)
                c.append_particles(k, sh.shed())
            c.sync()
            t1 = time.perf_counter()
            n_end = c.num_particles(k)
            import numpy as np
            amax = float(np.linalg.norm(c.state(k)[1], axis=1).max())
        print(f"rotor (omega {omega:g}, dt {sh.dt:.5f}): {steps} RK3 steps to {n_end} particles in {t1 - t0:.2f} s "
              f"({pairs:.3e} pairs, {pairs / (t1 - t0):.3e} pairs/s); last step {1e3 * (t1 - t_last):.1f} ms; "
              f"max |alpha| {amax:.3e}")


def merge_case(stations: int) -> None:
    import time
    w = cases.jittered(cases.ring_gaussian(stations=stations, per_section=1000, seed=1), 0.02, seed=1)
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.sync()
    t = time.perf_counter()
    m = c.merge(k, w.n)
    print(f"N {w.n} merge: {m} merges in {1e3 * (time.perf_counter() - t):.1f} ms")
    c.close()


def surrogate_case(n: int, solves: int) -> None:
    w = cases.leapfrog_rings(n_total=n)
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.surrogate_enable(order=2, tolerance=1e-4, check_targets=4096)
    for _ in range(solves):
        c.solve()
    c.sync()
    st = c.surrogate_stats()
    print(f"N {w.n} surrogate: tree {st['ms_tree']:.2f} ms, eval {st['ms_eval']:.2f} ms, check {st['ms_check']:.2f} ms, "
          f"sampled error {st['last_err_vel']:.2e}, fallbacks {st['fallbacks']}")
    c.close()


def mlp_case(steps: int) -> None:
    import numpy as np
    rng = np.random.default_rng(0)
    x = rng.normal(size=(262144, 24)).astype(np.float32)
    t = np.tanh(x[:, :6]).astype(np.float32)
    m = capi.Mlp(seed=1)
    m.set_dataset(x, t)
    hist = m.train(steps, batch=65536, lr=1e-3, seed=2)
    print(f"MLP {steps} training steps of batch 65536: loss {hist[0]:.4f} -> {hist[-1]:.4f}")


if __name__ == "__main__":
    main()
