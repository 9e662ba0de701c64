"""ctypes binding of the C ABI in ``include/pawan_gpu.h``.

The product path is ``lib/libpawan_gpu.so`` (built by ``pawan_b200.build``).
There is no CPU fallback: if the library or a GPU is missing, loading fails
with an exception.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

PGPU_OK = 0
PGPU_EINVAL = -1
PGPU_ENOMEM = -2
PGPU_ECUDA = -3
PGPU_ETIMEOUT = -4
PGPU_ENUMERIC = -5

FP32C = 0
FP64 = 1
# Regularisation kernels (PGPU_KERNEL_*): PAWAN's gaussian.h and highorder.h.
GAUSSIAN = 0
HIGHORDER = 1
KERNELS = {"gaussian": GAUSSIAN, "highorder": HIGHORDER}
EULER, RK3, RK4 = 0, 1, 2
SCHEMES = {"euler": EULER, "rk3": RK3, "rk4": RK4}

# Entry points declared in include/pawan_gpu.h (checked by the CPU tests).
EXPORTS = [
    "pgpu_config_default", "pgpu_create", "pgpu_destroy", "pgpu_add_wake", "pgpu_set_particles",
    "pgpu_append_particles", "pgpu_get_num_particles", "pgpu_get_state", "pgpu_set_states_flat",
    "pgpu_get_states_flat", "pgpu_get_rates_flat", "pgpu_solve", "pgpu_get_rates", "pgpu_step",
    "pgpu_diagnose", "pgpu_diagnose_partial", "pgpu_diagnose_combine", "pgpu_probe", "pgpu_sync", "pgpu_pair_kernel_time", "pgpu_launch_count",
    "pgpu_autotune", "pgpu_autotune_classes", "pgpu_kernel_shapes", "pgpu_last_error", "pgpu_version", "pgpu_get_stream",
    "pgpu_fp32_peak", "pgpu_fp32_peaks", "pgpu_fp64_peak", "pgpu_pair_counts", "pgpu_surrogate_config_default", "pgpu_surrogate_enable",
    "pgpu_surrogate_disable", "pgpu_surrogate_get_stats", "pgpu_surrogate_tree", "pgpu_mlp_num_params",
    "pgpu_mlp_create", "pgpu_mlp_destroy", "pgpu_mlp_last_error", "pgpu_mlp_get_params", "pgpu_mlp_set_params",
    "pgpu_mlp_forward", "pgpu_mlp_forward_fused", "pgpu_mlp_gradient", "pgpu_mlp_set_dataset", "pgpu_mlp_add_samples",
    "pgpu_mlp_dataset_rows", "pgpu_mlp_get_dataset", "pgpu_mlp_train", "pgpu_surrogate_set_mlp",
    "pgpu_rates_noalloc", "pgpu_noalloc_last_error", "pgpu_set_target_range", "pgpu_stage", "pgpu_records",
    "pgpu_sync_timeout", "pgpu_set_timing", "pgpu_influence", "pgpu_get_vorticity_field", "pgpu_merge",
    "pgpu_get_particles", "pgpu_snapshot_begin", "pgpu_snapshot_wait",
]


class PgpuConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("nu", C.c_double), ("vinf", C.c_double * 3),
                ("block", C.c_int), ("tpt", C.c_int), ("chunks", C.c_int), ("use_graphs", C.c_int),
                ("kernel", C.c_int), ("split_positions", C.c_int)]


class SurrogateConfig(C.Structure):
    _fields_ = [("leaf_size", C.c_int), ("near_widths", C.c_double), ("order", C.c_int), ("use_mlp", C.c_int),
                ("tolerance", C.c_double), ("check_targets", C.c_int), ("seed", C.c_int), ("far_u", C.c_double)]


class SurrogateStats(C.Structure):
    _fields_ = [("evaluations", C.c_int64), ("fallbacks", C.c_int64), ("last_err_vel", C.c_double),
                ("last_err_dalpha", C.c_double), ("max_err_vel", C.c_double), ("ms_tree", C.c_double),
                ("ms_eval", C.c_double), ("ms_check", C.c_double), ("ms_fallback", C.c_double),
                ("cells", C.c_int64), ("leaves", C.c_int64), ("far_entries", C.c_int64),
                ("near_entries", C.c_int64), ("max_err_dalpha", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneClass(C.Structure):
    _fields_ = [("size_class", C.c_int32), ("systems", C.c_int32), ("nmin", C.c_int64), ("nmax", C.c_int64),
                ("block", C.c_int32), ("tpt", C.c_int32), ("single_block", C.c_int32), ("single_tpt", C.c_int32),
                ("from_cache", C.c_int32), ("pad", C.c_int32), ("ms", C.c_double * 8)]


class PgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pawan_gpu error {code}: {msg}")
        self.code = code


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i64p = C.POINTER(C.c_int64)
_lib = None


def lib_path() -> Path:
    return _build.LIB


def load(build_if_missing: bool = False):
    """Loads libpawan_gpu.so (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not p.exists():
        if build_if_missing:
            _build.build()
        else:
            raise RuntimeError(f"{p} is missing: run `python -m pawan_b200.build`")
    lib = C.CDLL(str(p))
    vp = C.c_void_p
    sig = {
        "pgpu_config_default": (None, [C.POINTER(PgpuConfig)]),
        "pgpu_create": (C.c_int, [C.POINTER(vp), C.POINTER(PgpuConfig)]),
        "pgpu_destroy": (C.c_int, [vp]),
        "pgpu_add_wake": (C.c_int, [vp, C.c_int32, C.c_int64, C.POINTER(C.c_int32)]),
        "pgpu_set_particles": (C.c_int, [vp, C.c_int32, C.c_int64, _dp, _dp, _dp, _dp]),
        "pgpu_append_particles": (C.c_int, [vp, C.c_int32, C.c_int64, _dp, _dp, _dp, _dp]),
        "pgpu_get_num_particles": (C.c_int, [vp, C.c_int32, _i64p]),
        "pgpu_get_state": (C.c_int, [vp, C.c_int32, _dp, _dp]),
        "pgpu_set_states_flat": (C.c_int, [vp, _dp, _i64p, C.c_int32]),
        "pgpu_get_states_flat": (C.c_int, [vp, _dp, _i64p, C.c_int32]),
        "pgpu_get_rates_flat": (C.c_int, [vp, _dp, _i64p, C.c_int32]),
        "pgpu_solve": (C.c_int, [vp]),
        "pgpu_get_rates": (C.c_int, [vp, C.c_int32, _dp, _dp]),
        "pgpu_step": (C.c_int, [vp, C.c_int, C.c_double, C.c_int32]),
        "pgpu_diagnose": (C.c_int, [vp, C.c_int32, _dp, _dp]),
        "pgpu_diagnose_partial": (C.c_int, [vp, C.c_int32, _dp]),
        "pgpu_diagnose_combine": (C.c_int, [_dp, C.c_int32, C.c_double, _dp, _dp, _dp]),
        "pgpu_probe": (C.c_int, [vp, C.c_int32, C.c_int64, _dp, _dp]),
        "pgpu_sync": (C.c_int, [vp]),
        "pgpu_pair_kernel_time": (C.c_int, [vp, _dp, _i64p]),
        "pgpu_launch_count": (C.c_int64, [vp]),
        "pgpu_autotune": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
        "pgpu_kernel_shapes": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
        "pgpu_autotune_classes": (C.c_int, [vp, C.c_int, C.c_char_p, C.POINTER(TuneClass), C.c_int,
                                            C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "pgpu_last_error": (C.c_char_p, [vp]),
        "pgpu_version": (C.c_char_p, []),
        "pgpu_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "pgpu_fp32_peak": (C.c_int, [C.c_int, _dp, _dp]),
        "pgpu_fp32_peaks": (C.c_int, [C.c_int, _dp, _dp]),
        "pgpu_fp64_peak": (C.c_int, [C.c_int, _dp]),
        "pgpu_pair_counts": (C.c_int, [vp, _i64p, _i64p]),
        "pgpu_surrogate_config_default": (None, [C.POINTER(SurrogateConfig)]),
        "pgpu_surrogate_enable": (C.c_int, [vp, C.c_int32, C.POINTER(SurrogateConfig)]),
        "pgpu_surrogate_disable": (C.c_int, [vp]),
        "pgpu_surrogate_get_stats": (C.c_int, [vp, C.POINTER(SurrogateStats)]),
        "pgpu_mlp_num_params": (C.c_int, []),
        "pgpu_mlp_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int]),
        "pgpu_mlp_destroy": (C.c_int, [vp]),
        "pgpu_mlp_last_error": (C.c_char_p, [vp]),
        "pgpu_mlp_get_params": (C.c_int, [vp, _fp]),
        "pgpu_mlp_set_params": (C.c_int, [vp, _fp]),
        "pgpu_mlp_forward": (C.c_int, [vp, _fp, C.c_int64, _fp]),
        "pgpu_mlp_forward_fused": (C.c_int, [vp, _fp, C.c_int64, _fp]),
        "pgpu_mlp_gradient": (C.c_int, [vp, _fp, _fp, C.c_int64, _fp, _dp]),
        "pgpu_mlp_set_dataset": (C.c_int, [vp, _fp, _fp, C.c_int64]),
        "pgpu_mlp_add_samples": (C.c_int, [vp, vp, C.c_int64, C.c_int]),
        "pgpu_mlp_dataset_rows": (C.c_int64, [vp]),
        "pgpu_mlp_get_dataset": (C.c_int, [vp, _fp, _fp, C.c_int64]),
        "pgpu_mlp_train": (C.c_int, [vp, C.c_int, C.c_int, C.c_double, C.c_int, _fp]),
        "pgpu_surrogate_set_mlp": (C.c_int, [vp, vp]),
        "pgpu_surrogate_tree": (C.c_int, [vp, C.POINTER(C.c_int), C.c_int64, C.POINTER(C.c_int), C.c_int64,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int64, _i64p, _i64p, _i64p]),
        "pgpu_rates_noalloc": (C.c_int, [vp, vp, vp, vp, C.c_int64, C.c_double, vp, vp, vp]),
        "pgpu_noalloc_last_error": (C.c_char_p, []),
        "pgpu_set_target_range": (C.c_int, [vp, C.c_int32, C.c_int64, C.c_int64]),
        "pgpu_stage": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
        "pgpu_records": (C.c_int, [vp, C.c_int32, C.POINTER(vp), C.POINTER(vp)]),
        "pgpu_sync_timeout": (C.c_int, [vp, C.c_double]),
        "pgpu_set_timing": (C.c_int, [vp, C.c_int]),
        "pgpu_influence": (C.c_int, [vp]),
        "pgpu_get_vorticity_field": (C.c_int, [vp, C.c_int32, _dp]),
        "pgpu_merge": (C.c_int, [vp, C.c_int32, C.c_int64, _i64p]),
        "pgpu_get_particles": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp, _dp]),
        "pgpu_snapshot_begin": (C.c_int, [vp, C.c_int32]),
        "pgpu_snapshot_wait": (C.c_int, [vp, C.c_int32, C.c_double, C.POINTER(_dp), _i64p, _i64p, C.c_int32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def fp32_peaks(device: int = 0) -> tuple[float, float]:
    """Measured FP32 FMA throughput in TFLOP/s: (scalar FFMA loop, packed FFMA2 loop)."""
    lib = load()
    f1, f2 = C.c_double(), C.c_double()
    rc = lib.pgpu_fp32_peaks(device, C.byref(f1), C.byref(f2))
    if rc != PGPU_OK:
        raise PgpuError(rc, "pgpu_fp32_peaks failed")
    return f1.value, f2.value


def fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA throughput of the device in TFLOP/s (the larger of
    the scalar and packed loops)."""
    lib = load()
    tf, ms = C.c_double(), C.c_double()
    rc = lib.pgpu_fp32_peak(device, C.byref(tf), C.byref(ms))
    if rc != PGPU_OK:
        raise PgpuError(rc, "pgpu_fp32_peak failed")
    return tf.value


def fp64_peak(device: int = 0) -> float:
    """Measured FP64 FMA throughput of the device in TFLOP/s (DFMA register loop)."""
    lib = load()
    tf = C.c_double()
    rc = lib.pgpu_fp64_peak(device, C.byref(tf))
    if rc != PGPU_OK:
        raise PgpuError(rc, "pgpu_fp64_peak failed")
    return tf.value


DIAG_FIELDS = 23  # PGPU_DIAG_FIELDS


def diagnose_combine(fields, zc_prev: float = 0.0):
    """pgpu_diagnose_combine (host only): the 15-value diagnostics record, vbi
    and the new Zc from per-wake fields (wakes x DIAG_FIELDS) summed over the
    contexts that share a system."""
    lib = load()
    f = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1, DIAG_FIELDS)
    out, vbi, zc = np.zeros(15), np.zeros(3), C.c_double()
    rc = lib.pgpu_diagnose_combine(_p(f), f.shape[0], float(zc_prev), _p(out), _p(vbi), C.byref(zc))
    if rc != PGPU_OK:
        raise PgpuError(rc, "pgpu_diagnose_combine failed")
    return out, vbi, zc.value


NOALLOC_MAX_N = 32768  # PGPU_NOALLOC_MAX_N


def rates_noalloc(pos: int, alpha: int, sigma: int, vol: int, n: int, nu: float, vel: int, dalpha: int,
                  stream: int = 0) -> None:
    """pgpu_rates_noalloc on device addresses (row-major FP64 (n, 3) / (n,)
    arrays); queues the work on `stream` and returns without waiting."""
    lib = load()
    rc = lib.pgpu_rates_noalloc(pos, alpha, sigma, vol, n, nu, vel, dalpha, stream or None)
    if rc != PGPU_OK:
        raise PgpuError(rc, lib.pgpu_noalloc_last_error().decode())


def surrogate_config(**kw) -> SurrogateConfig:
    """pgpu_surrogate_config_default with the given fields replaced; an
    unknown field name is an error (a ctypes structure would otherwise keep
    it as a plain attribute that the library never sees)."""
    lib = load()
    cfg = SurrogateConfig()
    lib.pgpu_surrogate_config_default(C.byref(cfg))
    fields = {name for name, _ in SurrogateConfig._fields_}
    for k, v in kw.items():
        if k not in fields:
            raise TypeError(f"unknown surrogate setting {k!r} (fields: {', '.join(sorted(fields))})")
        setattr(cfg, k, v)
    return cfg


def wake_arrays(w) -> list[np.ndarray]:
    """Contiguous FP64 (pos, alpha, sigma, vol) of a wake of w.n particles.
    The library reads the first 3n, 3n, n and n values of them (row-major), so
    shorter arrays are rejected here instead of being over-read."""
    n = int(w.n)
    out = []
    for name, per in (("pos", 3), ("alpha", 3), ("sigma", 1), ("vol", 1)):
        a = _c(getattr(w, name))
        if a.size < per * n:
            raise ValueError(f"{name} holds {a.size} values; a wake of {n} particles needs {per * n}")
        out.append(a)
    return out


def kernel_shapes() -> list[tuple[int, int]]:
    lib = load()
    b = (C.c_int * 32)()
    t = (C.c_int * 32)()
    n = lib.pgpu_kernel_shapes(b, t, 32)
    return [(b[i], t[i]) for i in range(n)]


class Context:
    """One backend context: wakes grouped into systems, all device-resident."""

    def __init__(self, precision: int = FP32C, nu: float = 1.56e-5, device: int = 0, vinf=(0.0, 0.0, 0.0),
                 block: int = 0, tpt: int = 0, chunks: int = 0, use_graphs: bool = True, kernel: int = GAUSSIAN,
                 split_positions: bool = False):
        self.lib = load()
        cfg = PgpuConfig()
        self.lib.pgpu_config_default(C.byref(cfg))
        cfg.precision = precision
        cfg.device = device
        cfg.nu = nu
        for k in range(3):
            cfg.vinf[k] = float(vinf[k])
        cfg.block, cfg.tpt, cfg.chunks = block, tpt, chunks
        cfg.use_graphs = 1 if use_graphs else 0
        cfg.kernel = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        cfg.split_positions = 1 if split_positions else 0
        h = C.c_void_p()
        rc = self.lib.pgpu_create(C.byref(h), C.byref(cfg))
        if rc != PGPU_OK:
            raise PgpuError(rc, self.lib.pgpu_last_error(None).decode())
        self.h = h
        self.wake_sizes: list[int] = []
        self.wake_system: list[int] = []

    def _ck(self, rc: int):
        if rc != PGPU_OK:
            raise PgpuError(rc, self.lib.pgpu_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.pgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ wakes
    def add_wake(self, capacity: int, system: int = 0) -> int:
        wid = C.c_int32()
        self._ck(self.lib.pgpu_add_wake(self.h, system, int(capacity), C.byref(wid)))
        self.wake_sizes.append(0)
        self.wake_system.append(system)
        return wid.value

    def set_particles(self, wake: int, w):
        arr = wake_arrays(w)
        self._ck(self.lib.pgpu_set_particles(self.h, wake, w.n, *[_p(a) for a in arr]))
        self.wake_sizes[wake] = w.n

    def append_particles(self, wake: int, w):
        arr = wake_arrays(w)
        self._ck(self.lib.pgpu_append_particles(self.h, wake, w.n, *[_p(a) for a in arr]))
        self.wake_sizes[wake] += w.n

    def num_particles(self, wake: int) -> int:
        n = C.c_int64()
        self._ck(self.lib.pgpu_get_num_particles(self.h, wake, C.byref(n)))
        return n.value

    def state(self, wake: int = 0, out=None):
        n = self.num_particles(wake)
        if out is None:
            out = (np.zeros((n, 3)), np.zeros((n, 3)))
        for a in out:
            # written in place: contiguous FP64 with room for the wake's n rows
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size >= 3 * n):
                raise ValueError(f"state output arrays must be C-contiguous float64 with room for {3 * n} values")
        self._ck(self.lib.pgpu_get_state(self.h, wake, _p(out[0]), _p(out[1])))
        return out

    def rates(self, wake: int = 0):
        n = self.num_particles(wake)
        v, a = np.zeros((n, 3)), np.zeros((n, 3))
        self._ck(self.lib.pgpu_get_rates(self.h, wake, _p(v), _p(a)))
        return v, a

    # ------------------------------------------------------------ solve / step
    def solve(self):
        self._ck(self.lib.pgpu_solve(self.h))

    def step(self, scheme: str | int, dt: float, nsteps: int = 1):
        s = SCHEMES[scheme] if isinstance(scheme, str) else scheme
        self._ck(self.lib.pgpu_step(self.h, s, float(dt), int(nsteps)))

    def set_timing(self, on: bool):
        """Pair-kernel timing on (default; calls wait for their pair kernels) or off (calls only queue work)."""
        self._ck(self.lib.pgpu_set_timing(self.h, 1 if on else 0))

    def sync(self, timeout: float | None = None):
        """Waits for the queued work; with `timeout` (seconds) a host watchdog
        raises PgpuError(PGPU_ETIMEOUT) instead of waiting longer."""
        if timeout is None:
            self._ck(self.lib.pgpu_sync(self.h))
        else:
            self._ck(self.lib.pgpu_sync_timeout(self.h, float(timeout)))

    def snapshot_begin(self, slot: int):
        """Queues an asynchronous download of every wake's positions and
        strengths into snapshot `slot` (0 or 1) and returns at once; work
        queued afterwards overlaps the copy (pgpu_snapshot_begin)."""
        self._ck(self.lib.pgpu_snapshot_begin(self.h, int(slot)))

    def snapshot_wait(self, slot: int, timeout: float = 0.0) -> list[tuple[np.ndarray, np.ndarray]]:
        """Waits for snapshot `slot` (PgpuError(PGPU_ETIMEOUT) after `timeout`
        seconds if > 0) and returns per wake (positions (n, 3), strengths (n, 3)),
        copied out of the context's pinned buffer."""
        nw = len(self.wake_sizes)
        state = _dp()
        off = np.zeros(max(nw, 1), dtype=np.int64)
        n = np.zeros(max(nw, 1), dtype=np.int64)
        self._ck(self.lib.pgpu_snapshot_wait(self.h, int(slot), float(timeout), C.byref(state),
                                             off.ctypes.data_as(_i64p), n.ctypes.data_as(_i64p), nw))
        total = int((off[:nw] + n[:nw]).max()) if nw else 0
        buf = np.ctypeslib.as_array(state, shape=(6 * total,)) if total else np.zeros(0)
        out = []
        for w in range(nw):
            o, m = int(off[w]), int(n[w])
            out.append((buf[6 * o: 6 * o + 3 * m].reshape(m, 3).copy(),
                        buf[6 * o + 3 * m: 6 * o + 6 * m].reshape(m, 3).copy()))
        return out

    def merge(self, wake: int, n_elig: int) -> int:
        """PAWAN's particle merge (__wake::merge) over the wake's first n_elig
        particles (those old enough to merge); returns the number of merges."""
        m = C.c_int64(0)
        self._ck(self.lib.pgpu_merge(self.h, wake, int(n_elig), C.byref(m)))
        return int(m.value)

    def particles(self, wake: int = 0):
        """(pos, alpha, sigma, vol) of a wake."""
        n = self.num_particles(wake)
        pos, alpha = np.zeros((n, 3)), np.zeros((n, 3))
        sigma, vol = np.zeros(n), np.zeros(n)
        self._ck(self.lib.pgpu_get_particles(self.h, wake, _p(pos), _p(alpha), _p(sigma), _p(vol)))
        return pos, alpha, sigma, vol

    def vorticity_field(self, wake: int = 0) -> np.ndarray:
        """PAWAN's influence(): the vorticity field (n x 3) at the wake's particles
        from all particles of its system; computes the field of every system."""
        self._ck(self.lib.pgpu_influence(self.h))
        out = np.zeros((self.num_particles(wake), 3))
        self._ck(self.lib.pgpu_get_vorticity_field(self.h, wake, _p(out)))
        return out

    def diagnose(self, system: int = 0):
        out = np.zeros(15)
        vbi = np.zeros(3)
        self._ck(self.lib.pgpu_diagnose(self.h, system, _p(out), _p(vbi)))
        return out, vbi

    def diagnose_partial(self, system: int = 0) -> np.ndarray:
        """pgpu_diagnose_partial: this context's share of the diagnostic sums
        (its owned targets), one row of DIAG_FIELDS per wake of the system."""
        nw = sum(1 for s in self.wake_system if s == system)
        f = np.zeros((nw, DIAG_FIELDS))
        self._ck(self.lib.pgpu_diagnose_partial(self.h, system, _p(f)))
        return f

    def probe(self, pts, system: int = 0) -> np.ndarray:
        pts = _c(pts).reshape(-1, 3)
        vel = np.zeros_like(pts)
        self._ck(self.lib.pgpu_probe(self.h, system, pts.shape[0], _p(pts), _p(vel)))
        return vel

    def pair_kernel_time(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        self._ck(self.lib.pgpu_pair_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(self.lib.pgpu_get_stream(self.h, C.byref(s)))
        return int(s.value or 0)

    def pair_counts(self) -> tuple[int, int]:
        """(ordered pairs, full-formula pairs) evaluated since the last call."""
        p, f = C.c_int64(), C.c_int64()
        self._ck(self.lib.pgpu_pair_counts(self.h, C.byref(p), C.byref(f)))
        return p.value, f.value

    # ------------------------------------------------------------ far-field surrogate
    # ------------------------------------------------------------ sharding
    def set_target_range(self, system: int, first: int, count: int):
        """Owned targets [first, first + count) of the system; count < 0 restores all."""
        self._ck(self.lib.pgpu_set_target_range(self.h, system, int(first), int(count)))

    def stage(self, scheme: str, stage: int, dt: float):
        self._ck(self.lib.pgpu_stage(self.h, SCHEMES[scheme], int(stage), float(dt)))

    def records(self, system: int = 0) -> tuple[int, int]:
        """Device addresses of the system's source records P and Q."""
        P, Q = C.c_void_p(), C.c_void_p()
        self._ck(self.lib.pgpu_records(self.h, system, C.byref(P), C.byref(Q)))
        return P.value, Q.value

    def surrogate_enable(self, system: int = 0, **kw):
        cfg = surrogate_config(**kw)
        self._ck(self.lib.pgpu_surrogate_enable(self.h, system, C.byref(cfg)))

    def surrogate_disable(self):
        self._ck(self.lib.pgpu_surrogate_disable(self.h))

    def surrogate_stats(self) -> dict:
        st = SurrogateStats()
        self._ck(self.lib.pgpu_surrogate_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def surrogate_tree(self) -> dict:
        """Octree of the last surrogate evaluation (host copies)."""
        n, nc, nl = C.c_int64(), C.c_int64(), C.c_int64()
        ip = C.POINTER(C.c_int)
        self._ck(self.lib.pgpu_surrogate_tree(self.h, None, 0, None, 0, None, None, 0, C.byref(n), C.byref(nc),
                                              C.byref(nl)))
        idx = np.zeros(n.value, np.int32)
        cell = np.zeros((nc.value, 4), np.int32)
        leaves = np.zeros(nl.value, np.int32)
        counts = np.zeros((2, nl.value), np.int32)
        self._ck(self.lib.pgpu_surrogate_tree(self.h, idx.ctypes.data_as(ip), n.value, cell.ctypes.data_as(ip),
                                              nc.value, leaves.ctypes.data_as(ip), counts.ctypes.data_as(ip),
                                              nl.value, C.byref(n), C.byref(nc), C.byref(nl)))
        return {"idx": idx, "cells": cell, "leaves": leaves, "far": counts[0], "near": counts[1]}

    def surrogate_set_mlp(self, mlp: "Mlp"):
        self._ck(self.lib.pgpu_surrogate_set_mlp(self.h, mlp.h))

    def launch_count(self) -> int:
        return int(self.lib.pgpu_launch_count(self.h))

    def autotune(self, reps: int = 2):
        b, t = C.c_int(), C.c_int()
        ms = np.zeros(32)
        self._ck(self.lib.pgpu_autotune(self.h, reps, C.byref(b), C.byref(t), _p(ms)))
        shapes = kernel_shapes()
        return (b.value, t.value), {shapes[i]: float(ms[i]) for i in range(len(shapes))}

    def autotune_classes(self, reps: int = 2, cache: str | None = None) -> dict:
        """pgpu_autotune_classes: shapes per size class of the systems.
        Returns {"per_class": bool, "classes": [...]}, one dict per class with
        its particle range, systems, fastest shape, the single shape with the
        least total time, whether the times came from `cache`, and the time of
        one launch per shape."""
        out = (TuneClass * 32)()
        k, per = C.c_int(), C.c_int()
        self._ck(self.lib.pgpu_autotune_classes(self.h, reps, cache.encode() if cache else None, out, 32,
                                                C.byref(k), C.byref(per)))
        shapes = kernel_shapes()
        classes = []
        for i in range(k.value):
            o = out[i]
            classes.append({"class": o.size_class, "nmin": o.nmin, "nmax": o.nmax, "systems": o.systems,
                            "block": o.block, "tpt": o.tpt, "single_block": o.single_block,
                            "single_tpt": o.single_tpt, "from_cache": bool(o.from_cache),
                            "ms": {f"{b}x{t}": float(o.ms[j]) for j, (b, t) in enumerate(shapes)}})
        return {"per_class": bool(per.value), "classes": classes}

    # ------------------------------------------------------------ PAWAN flat state vector
    def set_states_flat(self, state, maxn):
        m = np.ascontiguousarray(maxn, dtype=np.int64)
        st = _c(state)
        if st.size < 6 * int(m.sum()):
            raise ValueError(f"the flat state holds {st.size} values; capacities {m.tolist()} need {6 * int(m.sum())}")
        self._ck(self.lib.pgpu_set_states_flat(self.h, _p(st), m.ctypes.data_as(_i64p), len(m)))

    def get_states_flat(self, maxn):
        m = np.ascontiguousarray(maxn, dtype=np.int64)
        st = np.zeros(int(6 * m.sum()))
        self._ck(self.lib.pgpu_get_states_flat(self.h, _p(st), m.ctypes.data_as(_i64p), len(m)))
        return st

    def get_rates_flat(self, maxn):
        m = np.ascontiguousarray(maxn, dtype=np.int64)
        st = np.zeros(int(6 * m.sum()))
        self._ck(self.lib.pgpu_get_rates_flat(self.h, _p(st), m.ctypes.data_as(_i64p), len(m)))
        return st


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


MLP_IN, MLP_OUT = 24, 6  # features per row in, outputs per row out


def _rows(a, cols: int, name: str) -> np.ndarray:
    """Contiguous FP32 (rows, cols) view of a; any other shape is an error,
    since the library reads rows x cols values."""
    a = _f32(a)
    if a.ndim != 2 or a.shape[1] != cols:
        raise ValueError(f"{name} must have shape (rows, {cols}), not {a.shape}")
    return a


class Mlp:
    """The far-field correction network (see include/pawan_gpu.h)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.pgpu_mlp_create(C.byref(h), device, seed)
        if rc != PGPU_OK:
            raise PgpuError(rc, "pgpu_mlp_create failed")
        self.h = h
        self.n_params = int(self.lib.pgpu_mlp_num_params())

    def _ck(self, rc: int):
        if rc != PGPU_OK:
            raise PgpuError(rc, self.lib.pgpu_mlp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.pgpu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        self._ck(self.lib.pgpu_mlp_get_params(self.h, p.ctypes.data_as(_fp)))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        if p.shape != (self.n_params,):
            raise ValueError(f"params must have shape ({self.n_params},), not {p.shape}")
        self._ck(self.lib.pgpu_mlp_set_params(self.h, p.ctypes.data_as(_fp)))

    def forward(self, x) -> np.ndarray:
        x = _rows(x, MLP_IN, "x")
        y = np.zeros((x.shape[0], MLP_OUT), np.float32)
        self._ck(self.lib.pgpu_mlp_forward(self.h, x.ctypes.data_as(_fp), x.shape[0], y.ctypes.data_as(_fp)))
        return y

    def forward_fused(self, x) -> np.ndarray:
        x = _rows(x, MLP_IN, "x")
        y = np.zeros((x.shape[0], MLP_OUT), np.float32)
        self._ck(self.lib.pgpu_mlp_forward_fused(self.h, x.ctypes.data_as(_fp), x.shape[0], y.ctypes.data_as(_fp)))
        return y

    def gradient(self, x, t):
        x, t = _rows(x, MLP_IN, "x"), _rows(t, MLP_OUT, "t")
        if t.shape[0] != x.shape[0]:
            raise ValueError(f"{x.shape[0]} feature rows but {t.shape[0]} target rows")
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        self._ck(self.lib.pgpu_mlp_gradient(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0],
                                            g.ctypes.data_as(_fp), C.byref(loss)))
        return loss.value, g

    def set_dataset(self, x, t):
        x, t = _rows(x, MLP_IN, "x"), _rows(t, MLP_OUT, "t")
        if t.shape[0] != x.shape[0]:
            raise ValueError(f"{x.shape[0]} feature rows but {t.shape[0]} target rows")
        self._ck(self.lib.pgpu_mlp_set_dataset(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0]))

    def add_samples(self, ctx: Context, n: int, seed: int = 0):
        self._ck(self.lib.pgpu_mlp_add_samples(self.h, ctx.h, int(n), int(seed)))

    @property
    def rows(self) -> int:
        return int(self.lib.pgpu_mlp_dataset_rows(self.h))

    def dataset(self, max_rows: int | None = None):
        n = self.rows if max_rows is None else min(max_rows, self.rows)
        x = np.zeros((n, MLP_IN), np.float32)
        t = np.zeros((n, MLP_OUT), np.float32)
        self._ck(self.lib.pgpu_mlp_get_dataset(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), n))
        return x, t

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        hist = np.zeros(max(steps, 1), np.float32)
        self._ck(self.lib.pgpu_mlp_train(self.h, int(steps), int(batch), float(lr), int(seed),
                                         hist.ctypes.data_as(_fp)))
        return hist[:steps]
