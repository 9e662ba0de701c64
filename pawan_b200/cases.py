"""Seeded particle layouts for the vortex-particle workloads.

Every generator returns host FP64 arrays in PAWAN's wake layout
(``src/wake/wake.h:49-54``): positions and strengths as row-major ``(n, 3)``,
smoothing radii and volumes as ``(n,)``.

The geometry follows PAWAN's ring generators in spirit (``src/wake/vring.cpp``:
strength along the ring tangent ``(-sin psi, cos psi, 0)``, ``vring.cpp:33-35``),
but the particle distributions are the ones the benchmark workloads specify:

* ``ring_stations``   - rings discretised as azimuthal stations times a fixed
  cross-section stencil (1 centre, 8 at a/2, 16 at a), Gaussian core weights.
* ``ring_gaussian``   - rings whose cross-section offsets are drawn from a
  normal distribution with standard deviation a/2, equal strength per particle.
* ``uneven_rings``    - many independent rings with log-uniform sizes.
* ``RotorShedder``    - a synthetic 4-blade tip-vortex shedder for growing wakes.
* ``leapfrog_rings``  - two coaxial rings (Gaussian cross-sections).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Wake:
    """Particles of one wake (PAWAN ``__wake``: position, vorticity, radius, volume)."""

    pos: np.ndarray
    alpha: np.ndarray
    sigma: np.ndarray
    vol: np.ndarray

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def copy(self) -> "Wake":
        return Wake(self.pos.copy(), self.alpha.copy(), self.sigma.copy(), self.vol.copy())

    @staticmethod
    def concat(wakes: list["Wake"]) -> "Wake":
        return Wake(np.concatenate([w.pos for w in wakes]), np.concatenate([w.alpha for w in wakes]),
                    np.concatenate([w.sigma for w in wakes]), np.concatenate([w.vol for w in wakes]))

    def subset(self, n: int) -> "Wake":
        return Wake(self.pos[:n].copy(), self.alpha[:n].copy(), self.sigma[:n].copy(), self.vol[:n].copy())


def _stencil25(a: float) -> tuple[np.ndarray, np.ndarray]:
    """(r, theta) of the 25-point cross-section: 1 centre, 8 at a/2, 16 at a."""
    r = [0.0] + [0.5 * a] * 8 + [a] * 16
    th = [0.0] + [2 * math.pi * m / 8 for m in range(8)] + [2 * math.pi * m / 16 for m in range(16)]
    return np.array(r), np.array(th)


def ring_stations(R: float = 1.0, gamma: float = 1.0, a: float = 0.1, stations: int = 200,
                  sigma: float = 0.1, jitter: float = 1e-3, seed: int | None = 0,
                  z0: float = 0.0) -> Wake:
    """Vortex ring as ``stations`` azimuthal stations x 25 particles per cross-section.

    Strength alpha = gamma * w_j * (R dpsi) * t(psi) with Gaussian core weights
    w_j = exp(-r_j^2 / (2 a^2)) normalised over the 25 points; volume
    R dpsi * pi a^2 / 25; positions jittered by U(-jitter, jitter) from
    ``numpy.random.default_rng(seed)``.  With the defaults this is the 5000
    particle single-ring case (R=1, Gamma=1, a=0.1, sigma=0.1).
    """
    r, th = _stencil25(a)
    w = np.exp(-r ** 2 / (2 * a * a))
    w /= w.sum()
    dpsi = 2 * math.pi / stations
    psi = dpsi * np.arange(stations)
    P = psi[:, None]
    rr = r[None, :]
    x = (R + rr * np.cos(th)[None, :]) * np.cos(P)
    y = (R + rr * np.cos(th)[None, :]) * np.sin(P)
    z = z0 + rr * np.sin(th)[None, :] + 0 * P
    pos = np.stack([x, y, z], -1).reshape(-1, 3)
    t = np.stack([-np.sin(psi), np.cos(psi), np.zeros_like(psi)], -1)
    alpha = (gamma * R * dpsi) * (w[None, :, None] * t[:, None, :])
    alpha = alpha.reshape(-1, 3)
    n = pos.shape[0]
    if jitter and seed is not None:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    vol = np.full(n, R * dpsi * math.pi * a * a / 25.0)
    return Wake(np.ascontiguousarray(pos), np.ascontiguousarray(alpha), np.full(n, float(sigma)), vol)


def ring_gaussian(R: float = 1.0, gamma: float = 1.0, a: float = 0.1, stations: int = 1000,
                  per_section: int = 1000, sigma: float = 0.02, seed: int = 1, z0: float = 0.0,
                  rng: np.random.Generator | None = None) -> Wake:
    """Vortex ring with normally distributed cross-section offsets.

    Each of ``stations`` azimuthal stations carries ``per_section`` particles
    whose (radial, axial) offsets are drawn from N(0, (a/2)^2); every particle
    carries gamma/per_section of the circulation, so the sampled density is the
    Gaussian core.  With the defaults this is the 1M-particle ring
    (1000 x 1000, sigma=0.02, seed 1).
    """
    if rng is None:
        rng = np.random.default_rng(seed)
    dpsi = 2 * math.pi / stations
    psi = np.repeat(dpsi * np.arange(stations), per_section)
    off = rng.normal(0.0, 0.5 * a, size=(stations * per_section, 2))
    rad = R + off[:, 0]
    pos = np.stack([rad * np.cos(psi), rad * np.sin(psi), z0 + off[:, 1]], -1)
    t = np.stack([-np.sin(psi), np.cos(psi), np.zeros_like(psi)], -1)
    alpha = (gamma * R * dpsi / per_section) * t
    n = pos.shape[0]
    vol = np.full(n, R * dpsi * math.pi * a * a / per_section)
    return Wake(np.ascontiguousarray(pos), np.ascontiguousarray(alpha), np.full(n, float(sigma)), vol)


def uneven_rings(count: int = 64, nmin: float = 2e3, nmax: float = 2e5, seed: int = 2,
                 scale: float = 1.0) -> list[Wake]:
    """``count`` independent rings with particle counts log-uniform in [nmin, nmax].

    R ~ U(0.5, 2), Gamma ~ U(0.5, 2), a = 0.1 R, sigma = a; 25 particles per
    cross-section and round(N/25) stations.  ``scale`` shrinks every count (for
    tests) while keeping the draw sequence.
    """
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = float(np.exp(rng.uniform(math.log(nmin), math.log(nmax))))
        R = float(rng.uniform(0.5, 2.0))
        G = float(rng.uniform(0.5, 2.0))
        a = 0.1 * R
        st = max(1, int(round(n * scale / 25.0)))
        out.append(ring_stations(R=R, gamma=G, a=a, stations=st, sigma=a, jitter=1e-3 * R,
                                 seed=int(rng.integers(0, 2 ** 31))))
    return out


def leapfrog_rings(n_total: int = 4_000_000, R1: float = 1.0, R2: float = 1.2, gamma: float = 1.0,
                   a: float = 0.1, sigma: float = 0.02, dz: float = 0.3, seed: int = 4) -> Wake:
    """Two coaxial rings (R1 at z=0, R2 at z=dz) with Gaussian cross-sections."""
    rng = np.random.default_rng(seed)
    half = n_total // 2
    per = 1000 if half >= 1_000_000 else max(25, int(round(math.sqrt(half))))
    st = max(1, half // per)
    w1 = ring_gaussian(R1, gamma, a, st, per, sigma, rng=rng, z0=0.0)
    w2 = ring_gaussian(R2, gamma, a, st, per, sigma, rng=rng, z0=dz)
    return Wake.concat([w1, w2])


@dataclass
class RotorShedder:
    """Synthetic rotor tip-vortex shedder for a growing wake.

    ``blades`` tip vortices of a rotor of radius ``radius`` turning by
    ``dpsi_deg`` per step at angular speed ``omega``, so dt = dpsi / omega
    (dpsi in radians; omega = 1 by default).  Each step every
    blade sheds ``per_blade`` particles spread along the tip-helix segment it
    swept during the step; the helix descends ``pitch`` per revolution.  Each
    particle carries Gamma times its segment length along the helix tangent,
    volume (segment length) * pi * core^2, and smoothing radius ``sigma``.
    """

    blades: int = 4
    radius: float = 1.0
    pitch: float = 0.1
    dpsi_deg: float = 10.0
    per_blade: int = 200
    gamma: float = 0.05
    core: float = 0.02
    sigma: float = 0.03
    inflow: tuple = (0.0, 0.0, -0.05)
    omega: float = 1.0
    step_index: int = field(default=0)

    @property
    def dt(self) -> float:
        return math.radians(self.dpsi_deg) / self.omega

    def shed(self) -> Wake:
        """Particles shed during the current step (advances the step counter)."""
        k = self.step_index
        dpsi = math.radians(self.dpsi_deg)
        m = self.per_blade
        frac = (np.arange(m) + 0.5) / m
        pos, alpha = [], []
        for b in range(self.blades):
            psi0 = k * dpsi + 2 * math.pi * b / self.blades
            psi = psi0 + frac * dpsi
            # the newest end (psi0 + dpsi) sits at the rotor plane; older points lie lower
            zz = -self.pitch * (psi0 + dpsi - psi) / (2 * math.pi)
            p = np.stack([self.radius * np.cos(psi), self.radius * np.sin(psi), zz], -1)
            tang = np.stack([-self.radius * np.sin(psi), self.radius * np.cos(psi),
                             np.full_like(psi, self.pitch / (2 * math.pi))], -1)
            seg = np.linalg.norm(tang, axis=1, keepdims=True) * (dpsi / m)
            tang = tang / np.linalg.norm(tang, axis=1, keepdims=True)
            pos.append(p)
            alpha.append(self.gamma * seg * tang)
        pos = np.concatenate(pos)
        alpha = np.concatenate(alpha)
        seglen = np.linalg.norm(alpha, axis=1) / self.gamma
        self.step_index += 1
        return Wake(pos, alpha, np.full(pos.shape[0], self.sigma), seglen * math.pi * self.core ** 2)


def _rotate(v: np.ndarray, axis: np.ndarray, theta: float) -> np.ndarray:
    axis = axis / np.linalg.norm(axis)
    return v * math.cos(theta) + np.cross(axis, v) * math.sin(theta) + axis * np.dot(axis, v) * (1 - math.cos(theta))


def merge_clusters(stations: int = 40, clusters: int = 150, chains: int = 10, seed: int = 0,
                   young: float = 0.2) -> tuple[Wake, int, np.ndarray]:
    """A wake for PAWAN's particle merge (``__wake::merge``, wake.cpp:112-159).

    A ``ring_stations`` ring with, around random ring particles, 1-3 extra
    particles each at 0.2-1.4 times the merge reach 0.125 (r_i + r_j), with
    strengths rotated by 0, 0.005, 0.02, 0.3, 1.5 or 3 rad (PAWAN merges when
    1 - cos >= 1e-4) and scaled by 0.3-4; 20 zero-strength particles; all of
    it shuffled.  In front of it, ``chains`` lines of 6 particles 0.2 r apart
    whose strengths are each perpendicular to the sum of the ones before: the
    head absorbs them one by one and ends up more than twice the merge reach
    from where it started.  Returns (wake, n_elig, active): PAWAN's loop visits
    particles while ``stepnum - active > 45``; with stepnum 100 the first
    n_elig = (1 - young) n particles qualify, the next one does not.
    """
    rng = np.random.default_rng(seed)
    b = ring_stations(stations=stations, seed=seed)
    r = float(b.sigma[0])
    reach = 0.25 * r
    P, A, S, V = [b.pos], [b.alpha], [b.sigma], [b.vol]
    for _ in range(clusters):
        i = rng.integers(b.n)
        for _ in range(rng.integers(1, 4)):
            off = rng.normal(size=3)
            off *= rng.uniform(0.2, 1.4) * reach / np.linalg.norm(off)
            th = float(rng.choice([0.0, 0.005, 0.02, 0.3, 1.5, 3.0]))
            a = _rotate(b.alpha[i], rng.normal(size=3), th) * rng.uniform(0.3, 4.0)
            P.append((b.pos[i] + off)[None]); A.append(a[None]); S.append([r]); V.append([b.vol[i]])
    for _ in range(20):
        i = rng.integers(b.n)
        P.append((b.pos[i] + 0.01 * r)[None]); A.append(np.zeros((1, 3))); S.append([r]); V.append([1e-4])
    pos, alpha = np.concatenate(P), np.concatenate(A)
    sig, vol = np.concatenate(S).astype(float), np.concatenate(V).astype(float)
    perm = rng.permutation(pos.shape[0])
    pos, alpha, sig, vol = pos[perm], alpha[perm], sig[perm], vol[perm]
    cp, ca = [], []
    for _ in range(chains):
        x0 = rng.uniform(-1.5, 1.5, 3) + np.array([0.0, 0.0, 2.0])
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        tot = rng.normal(size=3) * 1e-3
        cp.append(x0); ca.append(tot.copy())
        for k in range(1, 6):
            u = np.cross(tot, rng.normal(size=3))
            u *= 1e-2 / np.linalg.norm(u)
            cp.append(x0 + k * 0.2 * r * d); ca.append(u)
            tot = tot + u
    nc = len(cp)
    w = Wake(np.concatenate([np.array(cp).reshape(-1, 3), pos]), np.concatenate([np.array(ca).reshape(-1, 3), alpha]),
             np.concatenate([np.full(nc, r), sig]), np.concatenate([np.full(nc, 1e-4), vol]))
    n_elig = int((1.0 - young) * w.n)
    active = np.zeros(w.n)
    if n_elig < w.n:
        active[n_elig] = 90.0
        active[n_elig + 1:] = rng.choice([0.0, 90.0], w.n - n_elig - 1)
    return w, n_elig, active


def jittered(w: Wake, theta: float, seed: int = 0) -> Wake:
    """``w`` with every strength rotated by ``theta`` about a random axis."""
    rng = np.random.default_rng(seed)
    ax = rng.normal(size=w.alpha.shape)
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    a = w.alpha
    c, s = math.cos(theta), math.sin(theta)
    rot = a * c + np.cross(ax, a) * s + ax * (ax * a).sum(1, keepdims=True) * (1 - c)
    return Wake(w.pos.copy(), np.ascontiguousarray(rot), w.sigma.copy(), w.vol.copy())
