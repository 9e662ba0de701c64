"""One vortex system over several GPUs: targets partitioned, source records
exchanged once per RK stage.

Each rank (one process per GPU) holds the whole system in its own context and
owns a contiguous block of its targets (pgpu_set_target_range).  An RK step
runs stage by stage: ``pgpu_stage`` evaluates the owned targets' rates from
the source records of all particles and advances the owned particles (state
and records); then the owned records of every rank are all-gathered, so that
every rank holds all sources for the next stage.  That all-gather is the only
data exchange of the path: N x 32 B per stage in FP32C mode (128 MB at 4M),
against O(N^2 / ranks) pair work.

Two exchanges share one stepper:

* ``DistExchange``: torch.distributed (NCCL on GPUs, one backend per process;
  gloo works the same way with CPU tensors);
* ``LocalExchange``: several backends in one process (one context per GPU, or
  several contexts on one GPU), records copied device to device in order.

A backend is any object with ``stage(scheme, stage, dt)``, ``own_records()``
(the owned rows as a (chunk, 8) tensor, zero padded), ``set_records(parts)``
(one such tensor per rank, rank order), ``scope()`` (the stream context its
copies run in), ``state()`` and ``first`` / ``count`` / ``chunk`` / ``n`` /
``rank`` / ``world`` / ``device``.  ``GpuShard`` wraps a C-ABI context.
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi

STAGES = {"euler": 1, "rk3": 3, "rk4": 4}


def partition(n: int, world: int, rank: int) -> tuple[int, int, int]:
    """(first, count, chunk): contiguous blocks of ceil(n / world) targets."""
    chunk = -(-n // world) if n else 0
    first = min(rank * chunk, n)
    return first, max(0, min(chunk, n - first)), chunk


class _DeviceArray:
    """A device buffer of the library seen by torch without a copy (CUDA array interface)."""

    def __init__(self, ptr: int, shape: tuple[int, ...], typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class GpuShard:
    """One rank's context: the whole system, owning targets [first, first + count)."""

    def __init__(self, wake, rank: int, world: int, precision: int = capi.FP32C, nu: float = 1e-4,
                 device: int = 0, **cfg):
        self.rank, self.world, self.n = rank, world, wake.n
        self.first, self.count, self.chunk = partition(wake.n, world, rank)
        self.device = torch.device("cuda", device)
        self.ctx = capi.Context(precision=precision, nu=nu, device=device, **cfg)
        self.wake = self.ctx.add_wake(wake.n)
        self.ctx.set_particles(self.wake, wake)
        self.ctx.set_target_range(0, self.first, self.count)
        p, q = self.ctx.records(0)
        self.dtype = torch.float32 if precision == capi.FP32C else torch.float64
        ts = "<f4" if precision == capi.FP32C else "<f8"
        self.P = torch.as_tensor(_DeviceArray(p, (wake.n, 4), ts), device=self.device)
        self.Q = torch.as_tensor(_DeviceArray(q, (wake.n, 4), ts), device=self.device)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream(), device=self.device)
        self._own = torch.zeros((self.chunk, 8), dtype=self.dtype, device=self.device)

    def stage(self, scheme: str, stage: int, dt: float):
        self.ctx.stage(scheme, stage, dt)

    def scope(self):
        return torch.cuda.stream(self.stream)

    def own_records(self) -> torch.Tensor:
        f, c = self.first, self.count
        self._own[:c, :4].copy_(self.P[f:f + c])
        self._own[:c, 4:].copy_(self.Q[f:f + c])
        return self._own

    def set_records(self, parts: list[torch.Tensor]):
        for r, part in enumerate(parts):
            if r == self.rank:
                continue
            f, c, _ = partition(self.n, self.world, r)
            self.P[f:f + c].copy_(part[:c, :4])
            self.Q[f:f + c].copy_(part[:c, 4:])

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        """(pos, alpha) of all particles; only the owned rows are current."""
        return self.ctx.state(self.wake)

    def diag_fields(self) -> np.ndarray:
        """This rank's share of the diagnostic sums (pgpu_diagnose_partial)."""
        return self.ctx.diagnose_partial(0)

    def close(self):
        self.ctx.close()


def diagnose_dist(backend, zc_prev: float = 0.0, group=None):
    """PAWAN's diagnose of the sharded system on every rank: each rank's
    per-wake fields over its owned targets, summed by one all-reduce of
    wakes x DIAG_FIELDS doubles (about 20 per wake), then combined
    (pgpu_diagnose_combine).  Returns (record[15], vbi[3], zc)."""
    import torch.distributed as dist
    f = torch.as_tensor(backend.diag_fields(), dtype=torch.float64)
    f = f.to(backend.device) if backend.device.type == "cuda" else f
    dist.all_reduce(f, op=dist.ReduceOp.SUM, group=group)
    return capi.diagnose_combine(f.cpu().numpy(), zc_prev)


def diagnose_local(backends, zc_prev: float = 0.0):
    """The same for backends of one process: the fields summed on the host."""
    total = sum(b.diag_fields() for b in backends)
    return capi.diagnose_combine(total, zc_prev)


class DistExchange:
    """All-gather of the owned records over a torch.distributed group."""

    def __init__(self, backend, group=None):
        import torch.distributed as dist
        self.dist, self.b, self.group = dist, backend, group
        own = backend.own_records()
        self.parts = [torch.empty_like(own) for _ in range(backend.world)]

    def __call__(self):
        with self.b.scope():
            own = self.b.own_records()
            self.dist.all_gather(self.parts, own, group=self.group)
            self.b.set_records(self.parts)


class LocalExchange:
    """Exchange among backends of one process: every backend's owned rows are
    copied into every other backend, each copy ordered after the producing
    backend's stage and before the consuming backend's next stage."""

    def __init__(self, backends):
        self.bs = backends

    def __call__(self):
        parts = []
        for b in self.bs:
            with b.scope():
                parts.append(b.own_records().clone())
            b.stream.synchronize()
        for b in self.bs:
            with b.scope():
                b.set_records([p.to(b.device) for p in parts])


class ShardedStepper:
    """Steps backends stage by stage with an exchange after every stage."""

    def __init__(self, backends, exchange):
        self.bs = backends if isinstance(backends, (list, tuple)) else [backends]
        self.exchange = exchange

    def step(self, scheme: str, dt: float, nsteps: int = 1):
        for _ in range(nsteps):
            for s in range(STAGES[scheme]):
                for b in self.bs:
                    b.stage(scheme, s, dt)
                self.exchange()


class GraphedStepper:
    """One GpuShard's RK step (stage launches and the NCCL all-gather after
    each stage) captured once in a CUDA graph on the context's stream and
    replayed per step.  The capture uses thread-local mode, so the process
    group's own bookkeeping on other threads stays legal, and the library's
    pair-kernel timing is switched off (timing reads events on the host).
    Every rank captures and replays the same collectives in the same order.
    Call close() before destroying the process group."""

    def __init__(self, backend: "GpuShard", exchange: "DistExchange", scheme: str, dt: float):
        self.b, self.scheme, self.dt = backend, scheme, dt
        # the work plan and NCCL's communicator are set up outside the capture:
        # a rate evaluation (the state does not move) and one exchange of the
        # unchanged records
        backend.ctx.solve()
        exchange()
        torch.cuda.synchronize(backend.device)
        backend.ctx.set_timing(False)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=backend.stream, capture_error_mode="thread_local"):
            for s in range(STAGES[scheme]):
                backend.stage(scheme, s, dt)
                exchange()

    def step(self, nsteps: int = 1):
        with torch.cuda.stream(self.b.stream):
            for _ in range(nsteps):
                self.graph.replay()

    def close(self):
        if self.graph is not None:
            torch.cuda.synchronize(self.b.device)
            self.graph.reset()
            self.graph = None
            self.b.ctx.set_timing(True)


def gather_state(backends) -> tuple[np.ndarray, np.ndarray]:
    """Whole (pos, alpha) from the owned rows of local backends."""
    pos = alpha = None
    for b in backends:
        p, a = b.state()
        if pos is None:
            pos, alpha = np.empty_like(p), np.empty_like(a)
        pos[b.first:b.first + b.count] = p[b.first:b.first + b.count]
        alpha[b.first:b.first + b.count] = a[b.first:b.first + b.count]
    return pos, alpha


def gather_state_dist(backend, group=None) -> tuple[np.ndarray, np.ndarray]:
    """Whole (pos, alpha) on every rank, all-gathered from the owned rows."""
    import torch.distributed as dist
    p, a = backend.state()
    own = torch.zeros((backend.chunk, 6), dtype=torch.float64, device=backend.device)
    f, c = backend.first, backend.count
    own[:c, :3] = torch.as_tensor(p[f:f + c])
    own[:c, 3:] = torch.as_tensor(a[f:f + c])
    parts = [torch.empty_like(own) for _ in range(backend.world)]
    dist.all_gather(parts, own, group=group)
    full = torch.cat(parts)[:backend.n].cpu().numpy()
    return np.ascontiguousarray(full[:, :3]), np.ascontiguousarray(full[:, 3:])

