"""Benchmark of the B200 vortex-particle hot path (RK4 steps/s, pair-interactions/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --case kernel|surrogate|mlp-train|merge|ring5k|uneven64|rotor [options]

Workload (one GPU): a vortex ring of N = 1,000,000 particles (1000 azimuthal
stations x 1000 particles per cross-section, Gaussian cross-section offsets
with std a/2, R = 1, Gamma = 1, a = 0.1, sigma = 0.02, seed 1), viscosity
1e-4, classical RK4 with dt = 0.005, FP32 pair terms with compensated
per-target sums and FP64 state.  A step is one full RK4 step: four all-pairs
rate evaluations (4 x N (N - 1) ordered pair interactions) and the stage
updates.  Synthetic seeded data (no dataset is involved).

With --gpus N > 1 (torchrun, one rank per GPU) every rank advances its own
copy of the ring (independent replicas, weak scaling; the step has no
collective); --mode shard splits one ring's targets over the ranks instead.

`value` is RK4 steps/s with the particles resident in HBM (CUDA events on the
library's stream, max over ranks); `e2e` is the same metric through the C ABI
with host buffers: each step uploads the particles from pinned host memory,
steps, and downloads the new state.  `roofline` rates the pair kernel against
the FP32 FMA peak measured on the same GPU (the larger of a scalar FFMA and a
packed FFMA2 register loop); `cpu_baseline` times PAWAN's own OpenMP code
(compiled from its sources) on the host cores on a bounded sample and
extrapolates quadratically to N.

Sub-objects of the JSON line, measured after the headline timing in a
one-GPU run (N = 1; with N > 1 they and `cpu_baseline` are null, since they do
not change with N and the other GPUs would wait idle):
`fp64` (the same ring stepped in the FP64 mode, rated against the measured
FP64 FMA peak), `diagnostics` (one pgpu_diagnose of the ring), `uneven64` (64
independent rings of 2e3..2e5 particles in one persistent launch per stage,
shapes autotuned per size class) and `surrogate` (two coaxial rings of 4M
particles: the octree far field against the plain direct-sum RK4 step, with
a check of sampled targets against the FP64 restatement).

--impl reference runs PAWAN's own CPU implementation (oracle/_ref) on the
host cores with all threads: each step is one RK4 step of a random
SAMPLE_N-particle subset of the same ring, and the reported steps/s is
extrapolated to N by the ratio of pair counts.  The GPU arm's cpu_baseline
uses the same sample size and the same estimator (mean of timed steps).

--case runs one smaller workload for profilers (ncu) and quick timing; see
run_case.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_STATIONS, N_SECTION = 1000, 1000
SIGMA, NU, DT = 0.02, 1e-4, 0.005
FLOPS_PER_PAIR = 95  # algorithmic count of one ordered pair interaction (full formula)
FLOPS_PER_FAR_PAIR = 59  # same tally with erf = 1 and exp(-u/2) = 0 (far-field limit)
DIAG_FLOPS_PER_PAIR = 85  # helicity + KE + KEF per unordered pair (algorithmic count)
SAMPLE_N = 6000      # particles in the bounded CPU sample (both CPU legs)
CPU_SAMPLE_STEPS = 3  # timed sample steps of the GPU arm's cpu_baseline leg (after one untimed)
WORKLOAD = "vortex ring N=1M (1000 stations x 1000/section, gaussian core a=0.1, sigma=0.02), RK4 dt=0.005, FP32c pairs + FP64 state"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one pair-kernel
# launch from an ncu capture, keyed by (particles, block, targets per thread);
# reported as roofline.traffic only when the timed run used that shape.
NCU_TRAFFIC = {
    (1_000_000, 128, 2): (220_014_336, "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                                       "pair_kernel<float,128,2,128,0,0> on the 1M ring"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--stations", type=int, default=None,
                    help="azimuthal stations of the ring (default 1000 for the bench, 200 for --case)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the fp64, uneven64 and diagnostics sub-objects")
    ap.add_argument("--surrogate-n", type=int, default=4_000_000)
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="N > 1: every rank its own ring (replicas, weak scaling) or one ring with its targets "
                         "split over the ranks and the source records all-gathered per RK stage (shard, strong)")
    # --case options
    ap.add_argument("--case", default=None,
                    choices=["kernel", "surrogate", "mlp-train", "merge", "ring5k", "uneven64", "rotor"])
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--case-steps", type=int, default=1)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--block", type=int, default=0, help="pair-kernel block size (0: library default)")
    ap.add_argument("--tpt", type=int, default=0, help="targets per thread (0: library default)")
    ap.add_argument("--sigma", type=float, default=SIGMA, help="smoothing radius (smaller: fewer near pairs)")
    ap.add_argument("--kernel", choices=["gaussian", "highorder"], default="gaussian")
    ap.add_argument("--omega", type=float, default=1.0, help="rotor angular speed (dt = 10 deg / omega)")
    ap.add_argument("--mlp-steps", type=int, default=20)
    ap.add_argument("--report-every", type=int, default=0, help="rotor: a progress line every this many steps")
    ap.add_argument("--split", action="store_true", help="rotor: split FP32 positions (pgpu_config.split_positions)")
    a = ap.parse_args()
    if a.stations is None:
        a.stations = 200 if a.case else N_STATIONS
    return a


def workload(stations: int):
    from pawan_b200 import cases
    return cases.ring_gaussian(stations=stations, per_section=N_SECTION, sigma=SIGMA, seed=1)


def sample(w, n: int, seed: int = 0):
    from pawan_b200 import cases
    idx = np.sort(np.random.default_rng(seed).choice(w.n, n, replace=False))
    return cases.Wake(w.pos[idx], w.alpha[idx], w.sigma[idx], w.vol[idx])


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        load = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU reference
def reference_step_time(w, n: int) -> float:
    """Seconds of one RK4 step of PAWAN's own OpenMP code on an n-particle sample."""
    from oracle import oracle as O
    ws = sample(w, n)
    with O.quiet():
        R = O.RefSystem([ws], NU, parallel=True)
        lib = O.ref_lib()
        t0 = lib.ref_wtime()
        R.step("rk4", DT, 1)
        t = lib.ref_wtime() - t0
        R.close()
    return t


def extrapolate_steps_per_s(t_sample: float, n_sample: int, n: int) -> float:
    return 1.0 / (t_sample * (n * (n - 1)) / (n_sample * (n_sample - 1)))


def sample_desc(n_sample: int, n: int, steps: int) -> str:
    return (f"one RK4 step of PAWAN's own __parallel + __rk4 on a random {n_sample}-particle subset of the "
            f"{n}-particle ring, mean of {steps} timed steps after one untimed, extrapolated by pair count "
            f"N(N-1) to the whole ring")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpawanref.so was not built"}))
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    w = workload(args.stations)
    n = w.n
    for _ in range(max(args.warmup, 1)):
        reference_step_time(w, SAMPLE_N)
    times = [reference_step_time(w, SAMPLE_N) for _ in range(args.steps)]
    t = sum(times) / len(times)
    sps = extrapolate_steps_per_s(t, SAMPLE_N, n)
    cores = int(os.environ["OMP_NUM_THREADS"])
    out = {
        "metric": "RK4 steps/s", "value": sps, "unit": "steps/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": n, "sample_particles": SAMPLE_N,
                   "extrapolation": "steps/s x (n_s (n_s - 1)) / (N (N - 1))"},
        "pair_interactions_per_s": 4 * n * (n - 1) * sps,
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "reference",
                         "sample": sample_desc(SAMPLE_N, n, args.steps),
                         "sample_step_s": t},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def cpu_baseline_leg(w) -> dict | None:
    """PAWAN's own code on the host cores: the same sample size and estimator
    as the reference arm (one untimed step, then the mean of timed steps)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    reference_step_time(w, SAMPLE_N)
    t = sum(reference_step_time(w, SAMPLE_N) for _ in range(CPU_SAMPLE_STEPS)) / CPU_SAMPLE_STEPS
    return {"value": extrapolate_steps_per_s(t, SAMPLE_N, w.n), "unit": "steps/s",
            "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "reference",
            "sample": sample_desc(SAMPLE_N, w.n, CPU_SAMPLE_STEPS), "sample_step_s": t}


# ------------------------------------------------------------------ roofline helpers
def pair_roofline(pair_ms: float, launches: int, pairs: int, full: int, peak: float) -> dict:
    """Algorithmic TFLOP/s of the pair kernel under two flop conventions:
    95 flop per full-formula pair and 59 per far-limit pair (the pairs the
    kernel counted in each regime), and a flat 95 per ordered pair."""
    launches = max(launches, 1)
    avg_s = pair_ms / launches * 1e-3
    counted = (FLOPS_PER_PAIR * full + FLOPS_PER_FAR_PAIR * (pairs - full)) / launches / avg_s / 1e12
    flat = FLOPS_PER_PAIR * pairs / launches / avg_s / 1e12
    return {"achieved": counted, "frac": counted / peak, "achieved_flat95": flat, "frac_flat95": flat / peak,
            "pairs_per_s": pairs / launches / avg_s, "full_pair_fraction": full / max(pairs, 1),
            "pair_kernel_ms": pair_ms / launches}


def time_steps(ctx, stream, scheme: str, dt: float, steps: int, flush=None) -> float:
    """Device milliseconds of `steps` steps (CUDA events on the library's stream)."""
    import torch
    total = 0.0
    for i in range(steps):
        if i and flush is not None:
            flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(scheme, dt, 1)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total


# ------------------------------------------------------------------ sub-objects
def run_fp64(w, device: int, fp64_peak: float) -> dict:
    """The headline ring stepped in the FP64 mode (FP64 pair terms and state),
    one untimed and one timed RK4 step, shape 128 threads x 1 target (the FP64
    kernel's fastest at 1M: 3.09 s per evaluation against 3.22 s for 256 x 1
    and 3.6 s or more for the two- and four-target shapes)."""
    import torch
    from pawan_b200 import capi
    c = capi.Context(precision=capi.FP64, nu=NU, device=device, block=128, tpt=1)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    c.step("rk4", DT, 1)
    c.sync()
    c.pair_kernel_time()
    c.pair_counts()
    ms = time_steps(c, stream, "rk4", DT, 1)
    pair_ms, nl = c.pair_kernel_time()
    pairs, full = c.pair_counts()
    c.close()
    r = pair_roofline(pair_ms, nl, pairs, full, fp64_peak)
    return {"value": 1e3 / ms, "unit": "steps/s", "ms_per_step": ms, "steps": 1,
            "pair_interactions_per_s": 4 * w.n * (w.n - 1) / (ms * 1e-3),
            "roofline": {"bound": "fp64", "unit": "TFLOP/s", "peak": fp64_peak, **r,
                         "note": "95 flop per closed-form pair + 59 per far-limit pair (u >= 100, counted by the "
                                 "kernel) / CUDA-event launch time; peak = DFMA register loop measured on this GPU"}}


def run_uneven64(device: int, fp32_peak: float, steps: int = 3) -> dict:
    """64 independent rings (N log-uniform in [2e3, 2e5], seed 2) as 64
    systems of one context: one persistent pair launch per RK4 stage, the
    step replayed as a CUDA graph, shapes autotuned per size class."""
    import torch
    from pawan_b200 import capi, cases
    ws = cases.uneven_rings(count=64, nmin=2e3, nmax=2e5, seed=2)
    c = capi.Context(precision=capi.FP32C, nu=NU, device=device)
    ids = [c.add_wake(w.n, i) for i, w in enumerate(ws)]
    for i, w in zip(ids, ws):
        c.set_particles(i, w)
    tune = c.autotune_classes(reps=1)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    c.step("rk4", DT, 1)
    c.sync()
    c.pair_kernel_time()
    c.pair_counts()
    ms = time_steps(c, stream, "rk4", DT, steps)
    pair_ms, nl = c.pair_kernel_time()
    pairs, full = c.pair_counts()
    c.close()
    n = sum(w.n for w in ws)
    r = pair_roofline(pair_ms, nl, pairs, full, fp32_peak)
    return {"workload": "64 independent vortex rings, N log-uniform in [2e3, 2e5] (seed 2), R, Gamma ~ U(0.5, 2), "
                        "a = 0.1 R, sigma = a, RK4 dt=0.005, FP32c pairs + FP64 state",
            "particles": n, "value": steps / (ms * 1e-3), "unit": "steps/s", "ms_per_step": ms / steps,
            "steps": steps, "pair_interactions_per_s": pairs / (ms * 1e-3),
            "roofline": {"bound": "fp32", "unit": "TFLOP/s", "peak": fp32_peak, **r},
            "autotune": tune}


def run_diagnostics(ctx, stream, n: int, fp32_peak: float) -> dict:
    """One pgpu_diagnose of the ring after one warm call, CUDA events."""
    import torch
    ctx.diagnose(0)
    d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    d0.record(stream)
    ctx.diagnose(0)
    d1.record(stream)
    d1.synchronize()
    dms = d0.elapsed_time(d1)
    dflops = DIAG_FLOPS_PER_PAIR * n * (n - 1) / 2
    tf = dflops / (dms * 1e-3) / 1e12
    return {"ms": dms, "unordered_pairs": n * (n - 1) // 2, "achieved_tflops": tf, "frac": tf / fp32_peak,
            "note": f"{DIAG_FLOPS_PER_PAIR} flop per unordered pair (helicity 42 + KE 25 + KEF 18); "
                    "frac against the same FP32 peak as the step's roofline"}


def run_surrogate(args, device: int, shape, steps: int = 3, check_rows: int = 256) -> dict:
    """Two coaxial leapfrogging rings (R = 1 and 1.2, Gamma = 1, a = 0.1,
    sigma = 0.02, seed 4) of 4M particles.  One plain direct-sum RK4 step
    (autotuned pair-kernel shape of the 1M ring, the same kernel) against
    `steps` RK4 steps with the octree far field (quadrupole, near field within
    4 cell widths exact, 4096 sampled targets re-checked against the direct
    sum every evaluation, fallback if the velocity or dalpha/dt error passes
    1e-4), each timed whole after one untimed step.  Outside the timed region
    the surrogate's rates of `check_rows` seeded targets are compared with the
    oracle's FP64 restatement of PAWAN's pair sum."""
    import torch
    from oracle import oracle as O
    from pawan_b200 import capi, cases
    w = cases.leapfrog_rings(n_total=args.surrogate_n)
    out = {"workload": f"two coaxial rings N={w.n} (R=1, 1.2, Gamma=1, a=0.1, sigma=0.02, dz=0.3, seed 4), RK4 dt={DT}"}
    # plain direct-sum RK4 step
    c = capi.Context(precision=capi.FP32C, nu=NU, device=device, block=shape[0], tpt=shape[1])
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    direct_ms = time_steps(c, stream, "rk4", DT, 1)
    pair_ms, nl = c.pair_kernel_time()
    c.close()
    # surrogate steps from the same initial state
    c = capi.Context(precision=capi.FP32C, nu=NU, device=device, block=shape[0], tpt=shape[1])
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.surrogate_enable(order=2, tolerance=1e-4, check_targets=4096)
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    c.step("rk4", DT, 1)  # untimed (tree buffers)
    c.sync()
    sur_ms = time_steps(c, stream, "rk4", DT, steps)
    st = c.surrogate_stats()
    # the surrogate's rates at the current state against the FP64 restatement
    c.solve()
    vel, dal = c.rates(k)
    pos, alpha = c.state(k)
    c.close()
    rows = np.sort(np.random.default_rng(17).choice(w.n, check_rows, replace=False))
    now = cases.Wake(pos, alpha, w.sigma, w.vol)
    vr, ar = O.restate_rates(now, NU, targets=rows)
    ev, ea = O.rel_err(vel[rows], vr), O.rel_err(dal[rows], ar)
    direct_sps = 1e3 / direct_ms
    sur_sps = steps * 1e3 / sur_ms
    out.update({
        "direct_step_ms": direct_ms, "direct_pair_kernel_ms": pair_ms / max(nl, 1),
        "direct_shape": {"block": shape[0], "targets_per_thread": shape[1]},
        "surrogate_step_ms": sur_ms / steps, "surrogate_steps_timed": steps,
        "surrogate_steps_per_s": sur_sps, "direct_steps_per_s": direct_sps, "speedup": sur_sps / direct_sps,
        "sampled_rel_err_vel_max": st["max_err_vel"], "sampled_rel_err_dalpha_max": st["max_err_dalpha"],
        "fallbacks": st["fallbacks"], "evaluations": st["evaluations"], "far_order": 2,
        "learned_correction": False,
        "restatement_check": {"targets": check_rows, "rel_err_vel": ev, "rel_err_dalpha": ea,
                              "reference": "oracle FP64 restatement of PAWAN's pair sum (restate.c), host cores"},
        "tree": {"cells": st["cells"], "leaves": st["leaves"], "far_entries": st["far_entries"],
                 "near_runs": st["near_entries"]},
        "phase_ms_last_eval": {"tree": st["ms_tree"], "eval": st["ms_eval"], "check": st["ms_check"]}})
    return out


# ------------------------------------------------------------------ GPU arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    from pawan_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    w = workload(args.stations)
    n = w.n
    ctx = capi.Context(precision=capi.FP32C, nu=NU, device=local)
    k = ctx.add_wake(n)
    ctx.set_particles(k, w)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def l2_flush():
        with torch.cuda.stream(stream):
            flush.zero_()

    # the project's autotuner picks the pair-kernel shape for this size (untimed)
    shape, _ = ctx.autotune(reps=1)
    for _ in range(args.warmup):
        ctx.step("rk4", DT, 1)
    ctx.sync()
    ctx.pair_kernel_time()
    ctx.pair_counts()

    # ---- device-resident timing
    clocks = ClockSampler(local)
    launches0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    step_ms = time_steps(ctx, stream, "rk4", DT, args.steps, flush=l2_flush)
    ctx.sync()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    pair_ms, pair_launches = ctx.pair_kernel_time()
    pairs_timed, full_timed = ctx.pair_counts()
    t_ms = torch.tensor([step_ms], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    step_ms = float(t_ms.item())
    steps_per_s = args.steps / (step_ms * 1e-3)
    value = world * steps_per_s  # every rank advances its own ring
    pairs_per_launch = n * (n - 1)

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        hpos, halpha, hsig, hvol = pin((n, 3)), pin((n, 3)), pin((n,)), pin((n,))
        hpos[:], halpha[:], hsig[:], hvol[:] = w.pos, w.alpha, w.sigma, w.vol
        opos, oalpha = pin((n, 3)), pin((n, 3))
        from pawan_b200 import cases
        host = cases.Wake(hpos, halpha, hsig, hvol)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.set_particles(k, host)
            ctx.step("rk4", DT, 1)
            ctx.state(k, out=(opos, oalpha))
            hpos[:], halpha[:] = opos, oalpha
        e1.record(stream)
        e1.synchronize()
        e2e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
        if world > 1:
            dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
        e2e = {"value": world * args.steps / (float(e2e_ms.item()) * 1e-3), "unit": "steps/s",
               "h2d_bytes_per_step": int(hpos.nbytes + halpha.nbytes + hsig.nbytes + hvol.nbytes),
               "d2h_bytes_per_step": int(opos.nbytes + oalpha.nbytes),
               "wall_s": time.perf_counter() - t0}

    # the one-GPU sub-lines (diagnostics, FP64, 64 rings, surrogate) and the
    # CPU baseline run on rank 0 of a one-GPU run only: they do not change
    # with N, and the other GPUs would be held idle meanwhile
    extras = world == 1 and not args.no_extras
    diag = None
    if rank == 0:
        ffma_peak, ffma2_peak = capi.fp32_peaks(local)
        fp32_peak = max(ffma_peak, ffma2_peak)
        rl = pair_roofline(pair_ms, pair_launches, pairs_timed, full_timed, fp32_peak)
        diag = run_diagnostics(ctx, stream, n, fp32_peak) if extras else None
    ctx.close()
    fp64 = unev = sur = None
    if rank == 0 and extras:
        fp64 = run_fp64(w, local, capi.fp64_peak(local))
        unev = run_uneven64(local, fp32_peak)
    if rank == 0 and world == 1 and not args.no_surrogate:
        sur = run_surrogate(args, local, shape)

    if rank == 0:
        traffic = NCU_TRAFFIC.get((n, shape[0], shape[1]))
        cpu = cpu_baseline_leg(w) if world == 1 else None
        out = {
            "metric": "RK4 steps/s", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": n, "parallelism": f"replicas{world}",
                       "pair_kernel_shape": {"block": shape[0], "targets_per_thread": shape[1]},
                       "l2": "flushed between timed steps (256 MiB write)",
                       "precision": "FP32 pairs, compensated sums, FP64 state"},
            "pair_interactions_per_s": world * 4 * pairs_per_launch * steps_per_s,
            "pair_kernel_ms": rl["pair_kernel_ms"],
            "roofline": {"bound": "fp32", "achieved": rl["achieved"], "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": rl["frac"], "achieved_flat95": rl["achieved_flat95"],
                         "frac_flat95": rl["frac_flat95"],
                         "traffic": traffic[0] if traffic else None,
                         "traffic_source": traffic[1] if traffic else None,
                         "full_pair_fraction": rl["full_pair_fraction"],
                         "peak_ffma_loop": ffma_peak, "peak_ffma2_loop": ffma2_peak,
                         "note": f"frac: {FLOPS_PER_PAIR} flop per full-formula pair + {FLOPS_PER_FAR_PAIR} per "
                                 "far-limit pair (counted by the kernel); frac_flat95: 95 flop per ordered pair; "
                                 "both per launch / CUDA-event launch time; peak = the larger of a scalar FFMA "
                                 "and a packed FFMA2 register loop measured on this GPU (MEASURED_PEAKS.json has "
                                 "no FP32 figure)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "fp64": fp64,
            "diagnostics": diag,
            "uneven64": unev,
            "surrogate": sur,
        }
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


# ------------------------------------------------------------------ one ring over N GPUs
def run_shard(args):
    """--mode shard: the ring's targets split over the ranks (pawan_b200.shard),
    NCCL all-gather of the owned source records after every RK stage; value =
    RK4 steps/s of the one ring (strong scaling)."""
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from pawan_b200 import capi, shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29533")
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=timedelta(seconds=600),
                            device_id=torch.device("cuda", local))
    w = workload(args.stations)
    n = w.n
    b = shard.GpuShard(w, rank, world, precision=capi.FP32C, nu=NU, device=local)
    exchange = shard.DistExchange(b)
    stepper = shard.ShardedStepper(b, exchange)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    shape, _ = b.ctx.autotune(reps=1)  # over this rank's owned targets (untimed)
    b.ctx.pair_kernel_time()
    b.ctx.pair_counts()
    # eager warm-up steps: the pair kernel's device time and pair counts (the
    # graph replays below run with the library's timing off)
    for _ in range(args.warmup):
        stepper.step("rk4", DT, 1)
    torch.cuda.synchronize()
    pair_ms, pair_launches = b.ctx.pair_kernel_time()
    pairs_timed, full_timed = b.ctx.pair_counts()
    graphed = shard.GraphedStepper(b, exchange, "rk4", DT)
    graphed.step(1)  # first replay (untimed)
    clocks = ClockSampler(local)
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = 0.0
    for i in range(args.steps):
        if i:
            with torch.cuda.stream(b.stream):
                flush.zero_()
        ev0.record(b.stream)
        graphed.step(1)
        ev1.record(b.stream)
        ev1.synchronize()
        step_ms += ev0.elapsed_time(ev1)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    # per replayed step: per stage one box, one pair and one stage launch
    launches = args.steps * 4 * 3
    t = torch.tensor([step_ms], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms = float(t.item())
    steps_per_s = args.steps / (step_ms * 1e-3)

    e2e = None
    if not args.no_e2e:
        # each step: the whole ring from pinned host memory, the stage-by-stage
        # step with its exchanges, the owned rows back to the host
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        hpos, halpha, hsig, hvol = pin((n, 3)), pin((n, 3)), pin((n,)), pin((n,))
        hpos[:], halpha[:], hsig[:], hvol[:] = w.pos, w.alpha, w.sigma, w.vol
        from pawan_b200 import cases
        host = cases.Wake(hpos, halpha, hsig, hvol)
        opos, oalpha = pin((n, 3)), pin((n, 3))
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(b.stream)
        for _ in range(args.steps):
            b.ctx.set_particles(b.wake, host)
            graphed.step(1)
            b.ctx.state(b.wake, out=(opos, oalpha))
        e1.record(b.stream)
        e1.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": args.steps / (float(te.item()) * 1e-3), "unit": "steps/s",
               "h2d_bytes_per_step": int(hpos.nbytes + halpha.nbytes + hsig.nbytes + hvol.nbytes),
               "d2h_bytes_per_step": int(opos.nbytes + oalpha.nbytes)}

    if rank == 0:
        ffma_peak, ffma2_peak = capi.fp32_peaks(local)
        fp32_peak = max(ffma_peak, ffma2_peak)
        rl = pair_roofline(pair_ms, pair_launches, pairs_timed, full_timed, fp32_peak)
        out = {
            "metric": "RK4 steps/s", "value": steps_per_s, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": n, "parallelism": f"targets{world}",
                       "pair_kernel_shape": {"block": shape[0], "targets_per_thread": shape[1]},
                       "exchange": f"NCCL all-gather of the FP32 source records after each RK stage ({32 * n} B)",
                       "step": "stages and all-gathers of one RK4 step replayed from one CUDA graph",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "precision": "FP32 pairs, compensated sums, FP64 state"},
            "pair_interactions_per_s": 4 * n * (n - 1) * steps_per_s,
            "pair_kernel_ms": rl["pair_kernel_ms"],
            "roofline": {"bound": "fp32", "achieved": rl["achieved"], "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": rl["frac"], "frac_flat95": rl["frac_flat95"], "traffic": None,
                         "note": "rank 0's pair kernel over its owned targets; peak as in the replicas mode"},
            "cpu_baseline": None,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(out))
    graphed.close()  # the graph holds NCCL calls: released before the process group
    b.close()
    dist.destroy_process_group()


# ------------------------------------------------------------------ --case: workloads for profilers
def run_case(a) -> None:
    """One workload on cuda:0 through the C ABI, sized so that an ncu capture
    of one launch of its main kernel ends in about a minute:

    kernel     the bench ring geometry at `stations` x 1000 particles (200 ->
               N = 200,000): `solves` rate evaluations, `case-steps` RK4 steps
               and one diagnose; prints the pair-kernel time per launch
               (--fp64, --kernel, --block/--tpt, --sigma select variants)
    surrogate  the octree far field (order 2) on two coaxial rings of
               --surrogate-n particles, `solves` evaluations
    mlp-train  --mlp-steps training steps of the far-field network (batch 65536)
    merge      one particle merge (pgpu_merge) of the ring with strengths
               turned 0.02 rad
    ring5k     the 5000-particle ring (200 stations x 25, sigma 0.1, seed 0),
               RK4 dt = 0.01, FP64 and FP32C: device time of `case-steps`
               steps after one
    uneven64   64 independent rings with N log-uniform in [2e3, 2e5] (seed 2)
               as 64 systems of one context, RK4 dt = 0.005, FP32C, shapes
               autotuned per size class
    rotor      the growing 4-blade tip-vortex wake (200 particles per blade per
               step, 10 deg per step at angular speed --omega, RK3, inflow
               0.05 after each step, FP32C) for `case-steps` steps; reports the
               pair count, the time per step at the end and the largest
               strength (a bounded run keeps it near the shed strength)
    """
    from pawan_b200 import capi, cases
    name = a.case
    steps = max(a.case_steps, 1)
    if name == "kernel":
        w = cases.ring_gaussian(stations=a.stations, per_section=1000, sigma=a.sigma, seed=1)
        c = capi.Context(precision=capi.FP64 if a.fp64 else capi.FP32C, nu=NU, block=a.block, tpt=a.tpt,
                         kernel=a.kernel)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        for _ in range(a.solves):
            c.solve()
        c.sync()
        ms, nl = c.pair_kernel_time()
        pairs, full = c.pair_counts()
        per = ms / max(nl, 1)
        print(f"N {w.n} pair kernel {per:.3f} ms/launch, {w.n * (w.n - 1) / (per / 1e3):.3e} pairs/s, "
              f"full-formula fraction {full / max(pairs, 1):.4f}")
        if a.case_steps:
            c.step("rk4", DT, a.case_steps)
            c.sync()
        t = time.perf_counter()
        d, vbi = c.diagnose(0)
        print(f"diagnose {1e3 * (time.perf_counter() - t):.1f} ms; diagnostics", d.tolist(), "vbi", vbi.tolist())
        c.close()
    elif name == "surrogate":
        w = cases.leapfrog_rings(n_total=a.surrogate_n)
        c = capi.Context(precision=capi.FP32C, nu=NU)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.surrogate_enable(order=2, tolerance=1e-4, check_targets=4096)
        for _ in range(a.solves):
            c.solve()
        c.sync()
        st = c.surrogate_stats()
        print(f"N {w.n} surrogate: tree {st['ms_tree']:.2f} ms, eval {st['ms_eval']:.2f} ms, check "
              f"{st['ms_check']:.2f} ms, sampled error vel {st['last_err_vel']:.2e} dalpha {st['last_err_dalpha']:.2e}, "
              f"fallbacks {st['fallbacks']}")
        c.close()
    elif name == "mlp-train":
        rng = np.random.default_rng(0)
        x = rng.normal(size=(262144, 24)).astype(np.float32)
        t = np.tanh(x[:, :6]).astype(np.float32)
        m = capi.Mlp(seed=1)
        m.set_dataset(x, t)
        hist = m.train(a.mlp_steps, batch=65536, lr=1e-3, seed=2)
        print(f"MLP {a.mlp_steps} training steps of batch 65536: loss {hist[0]:.4f} -> {hist[-1]:.4f}")
    elif name == "merge":
        w = cases.jittered(cases.ring_gaussian(stations=a.stations, per_section=1000, seed=1), 0.02, seed=1)
        c = capi.Context(precision=capi.FP32C, nu=NU)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        c.sync()
        t = time.perf_counter()
        m = c.merge(k, w.n)
        print(f"N {w.n} merge: {m} merges in {1e3 * (time.perf_counter() - t):.1f} ms")
        c.close()
    elif name == "ring5k":
        w = cases.ring_stations(seed=0)
        for prec in (capi.FP64, capi.FP32C):
            with capi.Context(precision=prec, nu=NU) as c:
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
        import torch
        torch.cuda.set_device(0)
        fp32_peak = max(capi.fp32_peaks(0))
        print(json.dumps(run_uneven64(0, fp32_peak, steps)))
    else:
        sh = cases.RotorShedder(omega=a.omega)
        cap = 4 * sh.per_blade * (steps + 1)
        with capi.Context(precision=capi.FP32C, nu=NU, vinf=sh.inflow, split_positions=a.split) as c:
            k = c.add_wake(cap)
            first = sh.shed()
            c.set_particles(k, first)
            shed_sum = first.alpha.sum(axis=0)
            shed_abs = np.abs(first.alpha).sum()
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
                new = sh.shed()
                c.append_particles(k, new)
                shed_sum += new.alpha.sum(axis=0)
                shed_abs += np.abs(new.alpha).sum()
                if a.report_every and (it + 1) % a.report_every == 0:
                    c.sync()
                    _, alpha = c.state(k)
                    # stretching and diffusion are antisymmetric in each pair:
                    # the total strength equals the sum of the shed strengths
                    drift = float(np.abs(alpha.sum(axis=0) - shed_sum).max() / shed_abs)
                    print(json.dumps({"step": it + 1, "particles": c.num_particles(k),
                                      "elapsed_s": time.perf_counter() - t0, "pairs": pairs,
                                      "pairs_per_s": pairs / (time.perf_counter() - t0),
                                      "total_vorticity_drift": drift,
                                      "max_alpha": float(np.linalg.norm(alpha, axis=1).max())}), flush=True)
            c.sync()
            t1 = time.perf_counter()
            n_end = c.num_particles(k)
            amax = float(np.linalg.norm(c.state(k)[1], axis=1).max())
        print(f"rotor (omega {a.omega:g}, dt {sh.dt:.5f}): {steps} RK3 steps to {n_end} particles in {t1 - t0:.2f} s "
              f"({pairs:.3e} pairs, {pairs / (t1 - t0):.3e} pairs/s); last step {1e3 * (t1 - t_last):.1f} ms; "
              f"max |alpha| {amax:.3e}")


if __name__ == "__main__":
    a = parse()
    if a.case:
        run_case(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.mode == "shard":
        run_shard(a)
    else:
        run_ours(a)
