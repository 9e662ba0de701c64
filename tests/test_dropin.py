"""The C++ drop-in (pawan::__gpu, __rk4gpu, __rk3gpu) inside PAWAN's own time
loop __integration::integrate, against PAWAN's own __parallel + __rk4/__rk3.

The driver (tests/dropin/dropin_check.cpp) is compiled against PAWAN's headers
by tests/dropin/Makefile; it needs the PAWAN sources, so it is built where they
are and the binary is reused elsewhere.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import cases, wakeio

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"
DRIVER = ROOT / "tests" / "_build" / "dropin_check"
# the same driver built against PAWAN compiled with its high-order kernel
DRIVER_HO = ROOT / "tests" / "_build" / "dropin_check_ho"


@pytest.fixture(scope="module")
def driver():
    if not DRIVER.exists():
        pytest.skip("drop-in driver not built (make -C tests/dropin PAWAN_SRC=<PAWAN tree>)")
    return DRIVER


def run(driver, tmp_path, mode, scheme, w, dt, nsteps, nu=1e-4):
    pb = tmp_path / "particles.bin"
    wakeio.write_particles_bin(pb, w)
    out = tmp_path / f"{mode}_{scheme}"
    r = subprocess.run([str(driver), mode, scheme, str(pb), repr(dt), str(nsteps), str(out), repr(nu)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return wakeio.read_wake(str(out) + ".wake"), wakeio.read_diagnosis(str(out) + ".diagnosis")


def test_reader_on_reference_files():
    recs = wakeio.read_wake(GOLD / "integrate" / "ring1000_rk4.wake")
    assert len(recs) == 4
    assert [round(t, 12) for t, _ in recs] == [0.0, 0.01, 0.02, 0.03]
    assert all(len(ws) == 1 and ws[0].n == 1000 for _, ws in recs)
    nu, d = wakeio.read_diagnosis(GOLD / "integrate" / "ring1000_rk4.diagnosis")
    assert nu == 1e-4 and d.shape == (4, 16)
    g = np.load(GOLD / "ring1000.npz")
    np.testing.assert_allclose(d[0, 4:], g["diag"][3:], rtol=1e-10, atol=1e-14)
    assert O.rel_err(recs[2][1][0].pos, g["rk4_pos"]) < 1e-13


def test_writer_roundtrip(tmp_path):
    recs = wakeio.read_wake(GOLD / "integrate" / "ring1000_rk4.wake")
    p = tmp_path / "x.wake"
    with open(p, "wb") as f:
        for t, ws in recs:
            wakeio.write_wake_record(f, t, ws, ws[0].pos.shape[0])
    back = wakeio.read_wake(p)
    for (t0, a), (t1, b) in zip(recs, back):
        assert t0 == t1
        np.testing.assert_array_equal(a[0].pos, b[0].pos)
        np.testing.assert_array_equal(a[0].volume, b[0].volume)
    # byte-identical except the undefined high half of each maxN field
    raw0 = bytearray((GOLD / "integrate" / "ring1000_rk4.wake").read_bytes())
    raw1 = bytearray(p.read_bytes())
    rec = len(raw0) // 4
    for k in range(4):
        raw0[k * rec + 20: k * rec + 24] = b"\0\0\0\0"
    assert raw0 == raw1


def test_writer_rejects_rows_short_of_capacity(tmp_path):
    # PAWAN writes every capacity row of a wake; a record with fewer rows
    # would shift every later field of the file
    (t, ws), = wakeio.read_wake(GOLD / "integrate" / "ring1000_rk4.wake")[:1]
    maxn = ws[0].pos.shape[0]
    short = wakeio.WakeRecord(ws[0].n, ws[0].pos[:-1], ws[0].alpha, ws[0].radius, ws[0].active, ws[0].volume,
                              ws[0].birth)
    p = tmp_path / "short.wake"
    with open(p, "wb") as f:
        with pytest.raises(ValueError, match="pos has shape"):
            wakeio.write_wake_record(f, t, [short], maxn)
        too_many = wakeio.WakeRecord(maxn + 1, *[getattr(ws[0], k) for k in
                                                 ("pos", "alpha", "radius", "active", "volume", "birth")])
        with pytest.raises(ValueError, match="do not fit"):
            wakeio.write_wake_record(f, t, [too_many], maxn)
    assert p.stat().st_size == 0


def test_driver_reference_mode_reproduces_golden(driver, tmp_path, ref_available):
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    recs, (nu, d) = run(driver, tmp_path, "ref", "rk4", w, 0.01, 3)
    gold = wakeio.read_wake(GOLD / "integrate" / "ring1000_rk4.wake")
    _, gd = wakeio.read_diagnosis(GOLD / "integrate" / "ring1000_rk4.diagnosis")
    for (_, a), (_, b) in zip(recs, gold):
        assert O.rel_err(a[0].pos, b[0].pos) < 1e-13
        assert O.rel_err(a[0].alpha, b[0].alpha) < 1e-12
    np.testing.assert_allclose(d[:, 4:], gd[:, 4:], rtol=1e-10, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("gpu64", 1e-10), ("gpu", 1e-5)])
@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_dropin_matches_reference_in_pawan_time_loop(gpu, driver, tmp_path, ref_available, mode, tol, scheme):
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    ref, (_, dref) = run(driver, tmp_path, "ref", scheme, w, 0.01, 3)
    got, (nu, dgot) = run(driver, tmp_path, mode, scheme, w, 0.01, 3)
    assert nu == 1e-4 and len(got) == len(ref) == 4
    for (t0, a), (t1, b) in zip(got, ref):
        assert t0 == t1
        assert O.rel_err(a[0].pos, b[0].pos) < tol
        assert O.rel_err(a[0].alpha, b[0].alpha) < tol
    # diagnostics: O(N) impulses in FP64 on both sides; KE/KEF to the mode's tolerance
    np.testing.assert_allclose(dgot[:, 4:10], dref[:, 4:10], rtol=max(tol, 1e-10),
                               atol=max(tol, 1e-10) * np.abs(dref[:, 4:10]).max())
    np.testing.assert_allclose(dgot[:, 13:15], dref[:, 13:15], rtol=max(tol, 1e-10))


def _mask_maxn_high(raw: bytes, nrec: int) -> bytearray:
    """The .wake bytes with the undefined high half of each record's maxN
    field zeroed (interaction.cpp:311-312 writes an int with sizeof(size_t))."""
    b = bytearray(raw)
    rec = len(b) // nrec
    for k in range(nrec):
        b[k * rec + 20: k * rec + 24] = b"\0\0\0\0"
    return b


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("gpu64", 1e-10), ("gpu", 1e-5)])
@pytest.mark.parametrize("scheme", ["rk4", "rk3"])
def test_device_resident_integrate_writes_the_same_files(gpu, driver, tmp_path, ref_available, mode, tol, scheme):
    """__rk4gpu / __rk3gpu::integrate (state kept on the device, .wake records
    from asynchronous snapshots written by a thread) against PAWAN's own loop
    with the same GPU step: byte-identical .wake and .diagnosis files; and
    against PAWAN's __parallel + __rk4/__rk3 at the mode's tolerance."""
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    nsteps = 6
    ref, (_, dref) = run(driver, tmp_path, "ref", scheme, w, 0.01, nsteps)
    sync, _ = run(driver, tmp_path, mode, scheme, w, 0.01, nsteps)
    got, (nu, dgot) = run(driver, tmp_path, mode + "async", scheme, w, 0.01, nsteps)
    assert len(got) == len(sync) == len(ref) == nsteps + 1
    raw_sync = (tmp_path / f"{mode}_{scheme}.wake").read_bytes()
    raw_async = (tmp_path / f"{mode}async_{scheme}.wake").read_bytes()
    assert _mask_maxn_high(raw_async, nsteps + 1) == _mask_maxn_high(raw_sync, nsteps + 1)
    assert (tmp_path / f"{mode}async_{scheme}.diagnosis").read_bytes() == \
        (tmp_path / f"{mode}_{scheme}.diagnosis").read_bytes()
    for (t0, a), (t1, b) in zip(got, ref):
        assert t0 == t1
        assert O.rel_err(a[0].pos, b[0].pos) < tol
        assert O.rel_err(a[0].alpha, b[0].alpha) < tol
    np.testing.assert_allclose(dgot[:, 4:10], dref[:, 4:10], rtol=max(tol, 1e-10),
                               atol=max(tol, 1e-10) * np.abs(dref[:, 4:10]).max())


def _resolve(driver, out, backend):
    r = subprocess.run([str(driver), "resolve", backend, "3", "49", "0.1924", str(out)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.fromfile(str(out) + ".strengths")


@pytest.fixture(scope="module")
def resolved_ref(driver, tmp_path_factory):
    """PAWAN's strength solve __resolve::rebuild (resolve.cpp:12-63) on its own
    fusion-case ring __vring(1, 0.1, 3, 49, 0.1924), with __parallel."""
    if not O.ref_available():
        pytest.skip("oracle/_ref/libpawanref.so is not built (make -C oracle)")
    return _resolve(driver, tmp_path_factory.mktemp("resolve") / "ref", "ref")


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["gpu64", "gpu"])
def test_dropin_resolve_matches_reference(gpu, driver, resolved_ref, tmp_path, mode):
    """The same rebuild with __gpu: every column's influence() runs on the
    device, in FP64 in both modes; the solved strengths match PAWAN's.  The
    influence matrix's condition number (~1e6) turns the fields' last-digit
    differences into ~1e-9 of the strengths."""
    tol = 1e-8
    got = _resolve(driver, tmp_path / mode, mode)
    err = np.abs(got - resolved_ref).max() / np.abs(resolved_ref).max()
    print(f"resolve {mode}: max relative strength difference {err:.2e}")
    assert err < tol


@pytest.fixture(scope="module")
def driver_ho():
    if not DRIVER_HO.exists():
        pytest.skip("high-order drop-in driver not built (make -C tests/dropin all PAWAN_SRC=<PAWAN tree>)")
    return DRIVER_HO


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("gpu64", 1e-10), ("gpu", 1e-5)])
def test_dropin_highorder_build_matches_reference(gpu, driver_ho, tmp_path, ref_ho_available, mode, tol):
    """PAWAN built with highorder.h: __gpu picks the high-order kernel up from
    the build (pawan_kernel()) and matches __parallel + __rk4 of the same
    build in PAWAN's own time loop, enstrophy included."""
    g = np.load(GOLD / "ring1000.npz")
    w = cases.Wake(g["pos"], g["alpha"], g["sigma"], g["vol"])
    ref, (_, dref) = run(driver_ho, tmp_path, "ref", "rk4", w, 0.01, 3)
    got, (_, dgot) = run(driver_ho, tmp_path, mode, "rk4", w, 0.01, 3)
    gold = np.load(GOLD / "ring1000_ho.npz")
    # the reference run is the high-order one: its first diagnosis record is the fixture's
    np.testing.assert_allclose(dref[0, 4:], gold["diag"][3:], rtol=1e-10, atol=1e-14)
    for (t0, a), (t1, b) in zip(got, ref):
        assert t0 == t1
        assert O.rel_err(a[0].pos, b[0].pos) < tol
        assert O.rel_err(a[0].alpha, b[0].alpha) < tol
    # enstrophy, enstrophyF, KE, KEF
    np.testing.assert_allclose(dgot[:, 11:15], dref[:, 11:15], rtol=max(tol, 1e-10))


def _relax(driver, tmp_path, backend, w, ages, birth, stepnum):
    pb, ab = tmp_path / "particles.bin", tmp_path / "ages.bin"
    wakeio.write_particles_bin(pb, w)
    with open(ab, "wb") as f:
        np.array([w.n], dtype=np.int64).tofile(f)
        np.concatenate([ages, birth]).astype(np.float64).tofile(f)
    out = tmp_path / f"relax_{backend}"
    r = subprocess.run([str(driver), "relax", backend, str(pb), str(ab), str(stepnum), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    raw = np.fromfile(str(out) + ".relax")
    n = int(raw[:1].view(np.int64)[0])
    v = raw[1:]
    return n, v


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["gpu64", "gpu"])
def test_dropin_relax_matches_reference(gpu, driver, tmp_path, ref_available, mode):
    """PAWAN's relaxation __interaction::relax (split, then merge) through
    __gpu (split on the host wake, merge through pgpu_merge) against
    __parallel's, on a coupled-run wake layout: every array equal to the bit."""
    w, n_elig, active = cases.merge_clusters(seed=2)
    # a fifth of the eligible particles have grown to 2.5x their birth strength and split
    rng = np.random.default_rng(8)
    mag = np.linalg.norm(w.alpha, axis=1)
    birth = np.where(rng.random(w.n) < 0.2, mag / 2.5, mag)
    n_ref, ref = _relax(driver, tmp_path, "ref", w, active, birth, 100)
    n_got, got = _relax(driver, tmp_path, mode, w, active, birth, 100)
    assert n_got == n_ref > w.n  # split appended particles
    np.testing.assert_array_equal(got, ref)
