"""PAWAN's binary output formats: ``.wake`` and ``.diagnosis``.

Both are written by PAWAN's offline time loop ``__integration::integrate``
(src/integration/integration.cpp:96-132) and read by its post-processing
scripts (``scripts/readWake.py``, ``scripts/readDiagnostics.py``).

``.wake``: a sequence of records, one per written time, each
    t                      float64
    nWake                  uint64   (__interaction::write, interaction.cpp:306)
    maxN                   8 bytes: a C int written with sizeof(size_t)
                           (interaction.cpp:311-312) - only the low 4 bytes
                           are defined, the high 4 are whatever followed the
                           int in memory; readers take the low 4
    then per wake (__wake::write, wake.cpp:832-841):
    numParticles           uint64
    position, vorticity    maxN x 3 float64 each (all capacity rows)
    radius, active, volume, birthstrength   maxN float64 each

``.diagnosis``: nu (float64, __interaction::writenu), then per record
    t, total vorticity (3), linear impulse (3), angular impulse (3), helicity,
    enstrophy, enstrophyF, kinetic energy, kinetic energyF, Zc  (16 float64)
(integration.cpp:105-110, 122-126; interaction.cpp:321-335).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class WakeRecord:
    n: int
    pos: np.ndarray      # (maxN, 3)
    alpha: np.ndarray    # (maxN, 3)
    radius: np.ndarray   # (maxN,)
    active: np.ndarray
    volume: np.ndarray
    birth: np.ndarray


def read_wake(path) -> list[tuple[float, list[WakeRecord]]]:
    """All records of a .wake file: [(t, [WakeRecord per wake]), ...]."""
    buf = Path(path).read_bytes()
    off = 0
    out = []
    while off < len(buf):
        (t,) = struct.unpack_from("<d", buf, off)
        off += 8
        (nw,) = struct.unpack_from("<Q", buf, off)
        off += 8
        (maxn,) = struct.unpack_from("<i", buf, off)
        off += 8
        wakes = []
        for _ in range(nw):
            (n,) = struct.unpack_from("<Q", buf, off)
            off += 8
            arr = np.frombuffer(buf, dtype="<f8", count=maxn * 10, offset=off)
            off += 8 * maxn * 10
            pos = arr[: 3 * maxn].reshape(maxn, 3)
            alpha = arr[3 * maxn: 6 * maxn].reshape(maxn, 3)
            rest = arr[6 * maxn:].reshape(4, maxn)
            wakes.append(WakeRecord(int(n), pos, alpha, rest[0], rest[1], rest[2], rest[3]))
        out.append((t, wakes))
    return out


def read_diagnosis(path) -> tuple[float, np.ndarray]:
    """(nu, records (k, 16)) of a .diagnosis file; columns: t then the 15 diagnostics."""
    a = np.fromfile(path, dtype="<f8")
    return float(a[0]), a[1:].reshape(-1, 16)


def write_wake_record(f, t: float, wakes: list[WakeRecord], maxn: int) -> None:
    """Appends one .wake record (the high 4 bytes of the maxN field are written as 0).
    Every wake holds all maxN capacity rows, as PAWAN writes them; arrays of
    another length are rejected before anything is written."""
    for k, w in enumerate(wakes):
        shapes = {"pos": (maxn, 3), "alpha": (maxn, 3), "radius": (maxn,), "active": (maxn,), "volume": (maxn,),
                  "birth": (maxn,)}
        for name, shape in shapes.items():
            if np.shape(getattr(w, name)) != shape:
                raise ValueError(f"wake {k}: {name} has shape {np.shape(getattr(w, name))}, expected {shape}")
        if not 0 <= w.n <= maxn:
            raise ValueError(f"wake {k}: {w.n} particles do not fit {maxn} rows")
    f.write(struct.pack("<dQiI", t, len(wakes), maxn, 0))
    for w in wakes:
        f.write(struct.pack("<Q", w.n))
        for a in (w.pos, w.alpha, w.radius, w.active, w.volume, w.birth):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def write_diagnosis_header(f, nu: float) -> None:
    f.write(struct.pack("<d", nu))


def write_diagnosis_record(f, t: float, diag) -> None:
    f.write(struct.pack("<d", t))
    f.write(np.ascontiguousarray(diag, dtype="<f8").tobytes())


def write_particles_bin(path, w) -> None:
    """Particle file of the drop-in test driver: int64 n, then positions,
    strengths (n x 3 each), radii and volumes (n each), FP64."""
    with open(path, "wb") as f:
        f.write(struct.pack("<q", w.n))
        for a in (w.pos, w.alpha, w.sigma, w.vol):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
