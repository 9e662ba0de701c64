"""Benchmark of the B200 vortex-particle hot path (RK4 steps/s, pair-interactions/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): a vortex ring of N = 1,000,000 particles (1000 azimuthal
stations x 1000 particles per cross-section, Gaussian cross-section offsets
with std a/2, R = 1, Gamma = 1, a = 0.1, sigma = 0.02, seed 1), viscosity
1e-4, classical RK4 with dt = 0.005, FP32 pair terms with compensated
per-target sums and FP64 state.  A step is one full RK4 step: four all-pairs
rate evaluations (4 x N (N - 1) ordered pair interactions) and the stage
updates.  Synthetic seeded data (no dataset is involved).

With --gpus N > 1 (torchrun, one rank per GPU) every rank advances its own
copy of the ring (independent replicas, weak scaling; the step has no
collective).

`value` is RK4 steps/s with the particles resident in HBM (CUDA events on the
library's stream, max over ranks); `e2e` is the same metric through the C ABI
with host buffers: each step uploads the particles from pinned host memory,
steps, and downloads the new state.  `roofline` rates the pair kernel against
the FP32 FMA peak measured on the same GPU (the larger of a scalar FFMA and a
packed FFMA2 register loop); `cpu_baseline` times PAWAN's own
OpenMP code (compiled from its sources) on the host cores on a bounded sample
and extrapolates quadratically to N.

--impl reference runs PAWAN's own CPU implementation (oracle/_ref) on the
host cores with all threads: each step is one RK4 step of a random
SAMPLE_N-particle subset of the same ring, and the reported steps/s is
extrapolated to N by the ratio of pair counts.

The `surrogate` object times the far-field surrogate on rank 0: two coaxial rings of
4M particles, one RK4 step with the octree far field (quadrupole order,
sampled direct-sum check of 4096 targets per evaluation) against the plain
direct-sum RK4 step.
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
FLOPS_PER_FAR_PAIR = 59  # same tally with erf = 1 and exp(-u/2) = 0 (far-field limit, u >= 50)
DIAG_FLOPS_PER_PAIR = 85  # helicity + KE + KEF per unordered pair (algorithmic count)
SAMPLE_N = 4000      # particles in the bounded CPU sample
WORKLOAD = "vortex ring N=1M (1000 stations x 1000/section, gaussian core a=0.1, sigma=0.02), RK4 dt=0.005, FP32c pairs + FP64 state"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--stations", type=int, default=N_STATIONS, help="smaller rings for quick checks")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--surrogate-n", type=int, default=4_000_000)
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="N > 1: every rank its own ring (replicas, weak scaling) or one ring with its targets "
                         "split over the ranks and the source records all-gathered per RK stage (shard, strong)")
    return ap.parse_args()


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
def reference_step_time(w, n: int) -> tuple[float, int, str]:
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
    return t, os.cpu_count() or 1, f"one RK4 step of PAWAN __parallel + __rk4 on a random {n}-particle subset of the ring"


def extrapolate_steps_per_s(t_sample: float, n_sample: int, n: int) -> float:
    return 1.0 / (t_sample * (n * (n - 1)) / (n_sample * (n_sample - 1)))


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
    for _ in range(args.warmup):
        reference_step_time(w, SAMPLE_N)
    times = [reference_step_time(w, SAMPLE_N)[0] for _ in range(args.steps)]
    t = sum(times) / len(times)
    sps = extrapolate_steps_per_s(t, SAMPLE_N, n)
    cores = os.cpu_count() or 1
    out = {
        "metric": "RK4 steps/s", "value": sps, "unit": "steps/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": n, "sample_particles": SAMPLE_N,
                   "extrapolation": "steps/s x (n_s (n_s - 1)) / (N (N - 1))"},
        "pair_interactions_per_s": 4 * n * (n - 1) * sps,
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "reference",
                         "sample": f"one RK4 step of PAWAN's own __parallel/__rk4 on {SAMPLE_N} of the {n} particles, "
                                   f"mean of {args.steps}, extrapolated by pair count"},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


# ------------------------------------------------------------------ surrogate
def run_surrogate(args, device: int) -> dict:
    """Two coaxial leapfrogging rings (R = 1 and 1.2, Gamma = 1, a = 0.1,
    sigma = 0.02, seed 4): one RK4 step with the octree far field (quadrupole,
    near field within 4 cell widths exact, 4096 sampled targets re-checked
    against the direct sum every evaluation) against the plain direct sum.  The
    direct RK4 step is timed as four rate evaluations (its stage updates are
    ~1e-4 of it); the surrogate step is timed whole."""
    import torch
    from pawan_b200 import capi, cases
    w = cases.leapfrog_rings(n_total=args.surrogate_n)
    out = {"workload": f"two coaxial rings N={w.n} (R=1, 1.2, Gamma=1, a=0.1, sigma=0.02, dz=0.3, seed 4), RK4 dt={DT}"}
    c = capi.Context(precision=capi.FP32C, nu=NU, device=device)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.solve()
    c.sync()
    c.pair_kernel_time()
    c.solve()
    c.sync()
    direct_eval_ms, _ = c.pair_kernel_time()
    c.surrogate_enable(order=2, tolerance=1e-4, check_targets=4096)
    c.solve()  # warm-up (tree buffers)
    c.sync()
    stream = torch.cuda.ExternalStream(c.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    c.step("rk4", DT, 1)
    e1.record(stream)
    e1.synchronize()
    st = c.surrogate_stats()
    sur_ms = e0.elapsed_time(e1)
    direct_step_ms = 4 * direct_eval_ms
    out.update({"direct_eval_ms": direct_eval_ms, "direct_step_ms": direct_step_ms, "surrogate_step_ms": sur_ms,
                "surrogate_steps_per_s": 1e3 / sur_ms, "direct_steps_per_s": 1e3 / direct_step_ms,
                "speedup": direct_step_ms / sur_ms, "sampled_rel_err_vel_max": st["max_err_vel"],
                "sampled_rel_err_dalpha_last": st["last_err_dalpha"], "fallbacks": st["fallbacks"],
                "evaluations": st["evaluations"], "far_order": 2, "learned_correction": False,
                "tree": {"cells": st["cells"], "leaves": st["leaves"], "far_entries": st["far_entries"],
                         "near_runs": st["near_entries"]},
                "phase_ms_last_eval": {"tree": st["ms_tree"], "eval": st["ms_eval"], "check": st["ms_check"]}})
    c.close()
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
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms = 0.0
    for i in range(args.steps):
        if i:
            l2_flush()
        ev0.record(stream)
        ctx.step("rk4", DT, 1)
        ev1.record(stream)
        ev1.synchronize()
        step_ms += ev0.elapsed_time(ev1)
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
    pair_avg_ms = pair_ms / max(pair_launches, 1)

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

    # conserved-quantity diagnostics (pgpu_diagnose) of the same ring, outside
    # the timed region: one warm call, then one timed with CUDA events
    diag = None
    if rank == 0:
        ctx.diagnose(0)
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        d0.record(stream)
        ctx.diagnose(0)
        d1.record(stream)
        d1.synchronize()
        dms = d0.elapsed_time(d1)
        dflops = DIAG_FLOPS_PER_PAIR * n * (n - 1) / 2
        diag = {"ms": dms, "unordered_pairs": n * (n - 1) // 2,
                "achieved_tflops": dflops / (dms * 1e-3) / 1e12,
                "note": f"{DIAG_FLOPS_PER_PAIR} flop per unordered pair (helicity 42 + KE 25 + KEF 18); "
                        "frac against the same FP32 peak as the step's roofline"}

    sur = None
    if rank == 0 and not args.no_surrogate:
        ctx.close()
        sur = run_surrogate(args, local)

    if rank == 0:
        ffma_peak, ffma2_peak = capi.fp32_peaks(local)
        fp32_peak = max(ffma_peak, ffma2_peak)
        flops_per_launch = (FLOPS_PER_PAIR * full_timed + FLOPS_PER_FAR_PAIR * (pairs_timed - full_timed)) / max(pair_launches, 1)
        achieved = flops_per_launch / (pair_avg_ms * 1e-3) / 1e12
        # DRAM bytes of one pair-kernel launch at this size, from the ncu
        # capture summarised in profiles/ (a line "traffic_bytes_per_launch[N=..., ...] = B")
        traffic = None
        tf = ROOT / "profiles" / "pair_kernel_ring1M_dram.md"
        if tf.exists():
            import re
            for m in re.finditer(r"traffic_bytes_per_launch\[N=(\d+)[^\]]*\]\s*=\s*(\d+)", tf.read_text()):
                if int(m.group(1)) == n:
                    traffic = int(m.group(2))
        if diag is not None:
            diag["frac"] = diag["achieved_tflops"] / fp32_peak
        cpu = None
        from oracle import oracle as O
        if O.ref_available():
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
            t_s, cores, desc = reference_step_time(w, 6000)
            cpu = {"value": extrapolate_steps_per_s(t_s, 6000, n), "unit": "steps/s", "cores": cores,
                   "kind": "reference", "sample": desc + f" ({t_s:.1f} s), extrapolated by pair count to N={n}"}
        out = {
            "metric": "RK4 steps/s", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": n, "parallelism": f"replicas{world}",
                       "pair_kernel_shape": {"block": shape[0], "targets_per_thread": shape[1]},
                       "l2": "flushed between timed steps (256 MiB write)", "precision": "FP32 pairs, compensated sums, FP64 state"},
            "pair_interactions_per_s": world * 4 * pairs_per_launch * steps_per_s,
            "pair_kernel_ms": pair_avg_ms,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "traffic": traffic,
                         "full_pair_fraction": full_timed / max(pairs_timed, 1),
                         "peak_ffma_loop": ffma_peak, "peak_ffma2_loop": ffma2_peak,
                "note": f"{FLOPS_PER_PAIR} flop per full-formula pair + {FLOPS_PER_FAR_PAIR} per far-limit pair "
                        "(counted by the kernel) per launch / CUDA-event launch time; "
                        "peak = the larger of a scalar FFMA and a packed FFMA2 register loop measured on this GPU "
                        "(MEASURED_PEAKS.json has no FP32 figure)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "diagnostics": diag,
            "surrogate": sur,
        }
        print(json.dumps(out))
    if sur is None:
        ctx.close()
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
    stepper = shard.ShardedStepper(b, shard.DistExchange(b))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    shape, _ = b.ctx.autotune(reps=1)  # over this rank's owned targets (untimed)
    for _ in range(args.warmup):
        stepper.step("rk4", DT, 1)
    torch.cuda.synchronize()
    b.ctx.pair_kernel_time()
    b.ctx.pair_counts()
    clocks = ClockSampler(local)
    launches0 = b.ctx.launch_count()
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = 0.0
    for i in range(args.steps):
        if i:
            with torch.cuda.stream(b.stream):
                flush.zero_()
        ev0.record(b.stream)
        stepper.step("rk4", DT, 1)
        ev1.record(b.stream)
        ev1.synchronize()
        step_ms += ev0.elapsed_time(ev1)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    launches = b.ctx.launch_count() - launches0
    pair_ms, pair_launches = b.ctx.pair_kernel_time()
    pairs_timed, full_timed = b.ctx.pair_counts()
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
            stepper.step("rk4", DT, 1)
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
        pair_avg_ms = pair_ms / max(pair_launches, 1)
        flops_per_launch = (FLOPS_PER_PAIR * full_timed + FLOPS_PER_FAR_PAIR * (pairs_timed - full_timed)) / max(pair_launches, 1)
        achieved = flops_per_launch / (pair_avg_ms * 1e-3) / 1e12
        out = {
            "metric": "RK4 steps/s", "value": steps_per_s, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": n, "parallelism": f"targets{world}",
                       "pair_kernel_shape": {"block": shape[0], "targets_per_thread": shape[1]},
                       "exchange": f"NCCL all-gather of the FP32 source records after each RK stage ({32 * n} B)",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "precision": "FP32 pairs, compensated sums, FP64 state"},
            "pair_interactions_per_s": 4 * n * (n - 1) * steps_per_s,
            "pair_kernel_ms": pair_avg_ms,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "traffic": None,
                         "note": "rank 0's pair kernel over its owned targets; peak as in the replicas mode"},
            "cpu_baseline": None,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(out))
    b.close()
    dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.mode == "shard":
        run_shard(a)
    else:
        run_ours(a)
