"""CPU stand-in for pawan_b200.shard.GpuShard, for the multi-rank tests on
gloo: the same backend interface over FP64 numpy state, with the stage
arithmetic of the device's RK4 (rk4.cpp:12-77) and the owned targets' rates
from the oracle's FP64 restatement of PAWAN's pair sum.  Test code only."""
from __future__ import annotations

import contextlib

import numpy as np
import torch

from oracle import oracle as O
from pawan_b200 import cases
from pawan_b200.shard import partition


class CpuShard:
    def __init__(self, wake, rank: int, world: int, nu: float = 1e-4):
        self.rank, self.world, self.n, self.nu = rank, world, wake.n, nu
        self.first, self.count, self.chunk = partition(wake.n, world, rank)
        self.device = torch.device("cpu")
        self.sigma, self.vol = wake.sigma.copy(), wake.vol.copy()
        self.x0 = np.hstack([wake.pos, wake.alpha]).astype(np.float64)
        # records: stage state (pos, alpha) of every particle, sigma^2 / 2, volume
        self.rec = torch.tensor(np.hstack([self.x0, 0.5 * self.sigma[:, None] ** 2, self.vol[:, None]]))
        self.acc = np.zeros((self.count, 6))

    def scope(self):
        return contextlib.nullcontext()

    def stage(self, scheme: str, stage: int, dt: float):
        assert scheme == "rk4"
        f, c = self.first, self.count
        rec = self.rec.numpy()
        w = cases.Wake(rec[:, 0:3].copy(), rec[:, 3:6].copy(), self.sigma, self.vol)
        v, a = O.restate_rates(w, self.nu, targets=np.arange(f, f + c))
        k = np.hstack([v, a])
        x = self.x0[f:f + c]
        if stage == 0:
            self.acc = k.copy()
            y = x + 0.5 * dt * k
        elif stage == 1:
            self.acc += 2.0 * k
            y = x + 0.5 * dt * k
        elif stage == 2:
            self.acc += 2.0 * k
            y = x + dt * k
        else:
            self.x0[f:f + c] = x + (dt / 6.0) * (self.acc + k)
            y = self.x0[f:f + c]
        rec[f:f + c, 0:6] = y

    def own_records(self) -> torch.Tensor:
        out = torch.zeros((self.chunk, 8), dtype=torch.float64)
        out[:self.count] = self.rec[self.first:self.first + self.count]
        return out

    def set_records(self, parts):
        for r, part in enumerate(parts):
            if r == self.rank:
                continue
            f, c, _ = partition(self.n, self.world, r)
            self.rec[f:f + c] = part[:c]

    def state(self):
        return self.x0[:, :3].copy(), self.x0[:, 3:].copy()

    def diag_fields(self) -> np.ndarray:
        """The owned rows' share of the diagnostic sums from the oracle's FP64
        restatement, pair terms over every particle of the current records."""
        rec = self.rec.numpy()
        w = cases.Wake(rec[:, 0:3].copy(), rec[:, 3:6].copy(), self.sigma, self.vol)
        return O.restate_diagnose_fields(w, self.first, self.first + self.count)
