"""ctypes access to the parity oracle.  TEST INFRASTRUCTURE ONLY.

Two tiers, both built by ``oracle/Makefile`` into ``oracle/_ref/``:

* ``RefSystem`` drives PAWAN's own C++ classes (``__interaction`` /
  ``__parallel``, ``__rk3`` / ``__rk4``, ``__integration::integrate``) compiled
  from the unmodified PAWAN sources against the project's GSL-subset shim,
  once with PAWAN's default Gaussian kernel (``libpawanref.so``) and once with
  its high-order algebraic kernel (``libpawanref_ho.so``).
* ``restate_*`` call the FP64 CPU restatement (``oracle/restate.c``), validated
  against ``RefSystem`` at small N and used for sampled checks at large N.

Only ``tests/``, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _c(a, dtype=np.float64) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


_ref = {}
_rs = None
# Regularisation kernels, as the C ABI's PGPU_KERNEL_* values.
KERNELS = {"gaussian": 0, "highorder": 1}
_REF_LIBS = {0: "libpawanref.so", 1: "libpawanref_ho.so"}


def kernel_id(kernel) -> int:
    return KERNELS[kernel] if isinstance(kernel, str) else int(kernel)


@contextlib.contextmanager
def quiet():
    """Sends the process's stdout (file descriptor 1) to /dev/null: PAWAN's
    classes print progress with printf / std::cout."""
    libc = C.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def ref_available(kernel="gaussian") -> bool:
    return (REF_DIR / _REF_LIBS[kernel_id(kernel)]).exists()


def ref_lib(kernel="gaussian"):
    k = kernel_id(kernel)
    if k not in _ref:
        lib = C.CDLL(str(REF_DIR / _REF_LIBS[k]))
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int, _i64p, C.c_double, C.c_int]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_set_wake.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        lib.ref_get_wake.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        lib.ref_solve.argtypes = [C.c_void_p]
        lib.ref_get_rates.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        lib.ref_step.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        lib.ref_diagnose.argtypes = [C.c_void_p, _dp]
        lib.ref_getvi.argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_influence.argtypes = [C.c_void_p, _dp]
        lib.ref_integrate.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_char_p]
        lib.ref_merge.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int64]
        lib.ref_get_particles.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        lib.ref_wtime.restype = C.c_double
        _ref[k] = lib
    return _ref[k]


SCHEMES = {"euler": 0, "rk3": 1, "rk4": 2}


class RefSystem:
    """One PAWAN ``__interaction`` (or ``__parallel``) holding several wakes,
    from the PAWAN build of the given regularisation kernel."""

    def __init__(self, wakes, nu: float, parallel: bool = True, kernel="gaussian"):
        self.lib = ref_lib(kernel)
        self.ns = [w.n for w in wakes]
        n = np.array(self.ns, dtype=np.int64)
        self.h = self.lib.ref_create(len(wakes), n.ctypes.data_as(_i64p), float(nu), 1 if parallel else 0)
        self._keep = []
        for i, w in enumerate(wakes):
            arrs = [_c(w.pos), _c(w.alpha), _c(w.sigma), _c(w.vol)]
            self.lib.ref_set_wake(self.h, i, *[_p(a) for a in arrs])

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self):
        self.lib.ref_solve(self.h)

    def rates(self, w: int = 0):
        v = np.zeros((self.ns[w], 3))
        a = np.zeros((self.ns[w], 3))
        self.lib.ref_get_rates(self.h, w, _p(v), _p(a))
        return v, a

    def state(self, w: int = 0):
        x = np.zeros((self.ns[w], 3))
        a = np.zeros((self.ns[w], 3))
        self.lib.ref_get_wake(self.h, w, _p(x), _p(a))
        return x, a

    def step(self, scheme: str, dt: float, nsteps: int = 1):
        self.lib.ref_step(self.h, SCHEMES[scheme], float(dt), int(nsteps))

    def diagnose(self) -> np.ndarray:
        out = np.zeros(15)
        self.lib.ref_diagnose(self.h, _p(out))
        return out

    def vorticity_field(self) -> np.ndarray:
        """PAWAN's resolve()/influence(): the vorticity field of every particle,
        wakes concatenated in order (sum(ns) x 3)."""
        out = np.zeros((int(sum(self.ns)), 3))
        self.lib.ref_influence(self.h, _p(out))
        return out

    def getvi(self, r) -> np.ndarray:
        r = _c(r)
        out = np.zeros(3)
        self.lib.ref_getvi(self.h, _p(r), _p(out))
        return out

    def merge(self, w: int, active, stepnum: int):
        """PAWAN's __wake::merge on wake w with birth steps ``active``."""
        a = _c(active)
        self.lib.ref_merge(self.h, w, _p(a), int(stepnum))

    def particles(self, w: int = 0):
        n = self.ns[w]
        x, a, r, v = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n)
        self.lib.ref_get_particles(self.h, w, _p(x), _p(a), _p(r), _p(v))
        return x, a, r, v

    def integrate(self, scheme: str, t: float, n: int, diagnose: bool, path: str):
        self.lib.ref_integrate(self.h, SCHEMES[scheme], float(t), int(n), int(diagnose), str(path).encode())


def restate_lib():
    global _rs
    if _rs is None:
        lib = C.CDLL(str(REF_DIR / "librestate.so"))
        lib.rs_rates.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, _i64p, C.c_int64, _dp, _dp]
        lib.rs_step.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int64, _dp, _dp, _dp, _dp, C.c_double]
        lib.rs_diagnose.argtypes = [C.c_int, _i64p, _dp, _dp, _dp, C.c_double, _dp, _dp]
        lib.rs_getvi.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp]
        lib.rs_vorticity_field.argtypes = [C.c_int64, _dp, _dp, _dp, _i64p, C.c_int64, _dp]
        lib.rs_set_kernel.argtypes = [C.c_int]
        lib.rs_merge.argtypes = [C.c_int64, C.c_int64, _dp, _dp, _dp, _dp]
        lib.rs_merge.restype = C.c_int64
        lib.rs_threads.restype = C.c_int
        _rs = lib
    return _rs


def _restate(kernel):
    """The restatement library with its kernel switched to ``kernel``."""
    lib = restate_lib()
    lib.rs_set_kernel(kernel_id(kernel))
    return lib


def restate_rates(w, nu: float, targets=None, kernel="gaussian"):
    """(vel, dalpha) of the listed targets (all if None) from all particles of ``w``."""
    lib = _restate(kernel)
    pos, al, sg, vo = _c(w.pos), _c(w.alpha), _c(w.sigma), _c(w.vol)
    if targets is None:
        nt = w.n
        tp = None
    else:
        t = _c(targets, np.int64)
        nt = t.shape[0]
        tp = t.ctypes.data_as(_i64p)
    v = np.zeros((nt, 3))
    a = np.zeros((nt, 3))
    lib.rs_rates(w.n, _p(pos), _p(al), _p(sg), _p(vo), float(nu), tp, nt, _p(v), _p(a))
    return v, a


def restate_vorticity_field(w, targets=None, kernel="gaussian") -> np.ndarray:
    """Vorticity field (n x 3) of the listed targets (all if None) from all particles of ``w``."""
    lib = _restate(kernel)
    pos, al, sg = _c(w.pos), _c(w.alpha), _c(w.sigma)
    if targets is None:
        nt, tp = w.n, None
    else:
        t = _c(targets, np.int64)
        nt, tp = t.shape[0], t.ctypes.data_as(_i64p)
    out = np.zeros((nt, 3))
    lib.rs_vorticity_field(w.n, _p(pos), _p(al), _p(sg), tp, nt, _p(out))
    return out


def restate_step(w, nu: float, scheme: str, dt: float, nsteps: int, kernel="gaussian"):
    """Returns a new (pos, alpha) after ``nsteps`` steps."""
    lib = _restate(kernel)
    pos, al = _c(w.pos).copy(), _c(w.alpha).copy()
    sg, vo = _c(w.sigma), _c(w.vol)
    lib.rs_step(SCHEMES[scheme], float(dt), int(nsteps), w.n, _p(pos), _p(al), _p(sg), _p(vo), float(nu))
    return pos, al


def restate_diagnose(w, offsets=None, zc_prev: float = 0.0, kernel="gaussian"):
    lib = _restate(kernel)
    if offsets is None:
        offsets = [0, w.n]
    off = _c(offsets, np.int64)
    out = np.zeros(15)
    vbi = np.zeros(3)
    lib.rs_diagnose(len(offsets) - 1, off.ctypes.data_as(_i64p), _p(_c(w.pos)), _p(_c(w.alpha)),
                    _p(_c(w.sigma)), float(zc_prev), _p(out), _p(vbi))
    return out, vbi


def restate_getvi(w, r, kernel="gaussian") -> np.ndarray:
    """Velocity induced at point ``r`` by all particles of ``w``, each with its
    own radius (PAWAN's getVi)."""
    lib = _restate(kernel)
    out = np.zeros(3)
    lib.rs_getvi(w.n, _p(_c(w.pos)), _p(_c(w.alpha)), _p(_c(w.sigma)), _p(_c(r)), _p(out))
    return out


def restate_merge(w, n_elig: int):
    """PAWAN's particle merge over the first n_elig particles of ``w``:
    returns (pos, alpha, vol, merges), new arrays."""
    lib = restate_lib()
    pos, al, vo = _c(w.pos).copy(), _c(w.alpha).copy(), _c(w.vol).copy()
    m = lib.rs_merge(w.n, int(n_elig), _p(pos), _p(al), _p(_c(w.sigma)), _p(vo))
    return pos, al, vo, int(m)


def restate_threads() -> int:
    return int(restate_lib().rs_threads())


def rel_err(x, ref) -> float:
    """max_i |x_i - ref_i| / max_i |ref_i| over rows (infinity-norm relative error)."""
    x = np.asarray(x, dtype=np.float64).reshape(len(ref), -1) if np.ndim(ref) > 1 else np.asarray(x, np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.ndim == 1:
        den = np.max(np.abs(ref))
        return float(np.max(np.abs(x - ref)) / den) if den > 0 else float(np.max(np.abs(x - ref)))
    num = np.max(np.linalg.norm(x - ref, axis=1))
    den = np.max(np.linalg.norm(ref, axis=1))
    return float(num / den) if den > 0 else float(num)


def restate_diagnose_fields(w, row_lo: int, row_hi: int, offsets=None, kernel="gaussian") -> np.ndarray:
    """Per-wake diagnostic sums over the rows [row_lo, row_hi) in the C ABI's
    pgpu_diagnose_partial layout, shape (wakes, 23)."""
    lib = _restate(kernel)
    if not hasattr(lib, "_fields_bound"):
        lib.rs_diagnose_fields.argtypes = [C.c_int, _i64p, _dp, _dp, _dp, C.c_int64, C.c_int64, _dp]
        lib._fields_bound = True
    if offsets is None:
        offsets = [0, w.n]
    off = _c(offsets, np.int64)
    out = np.zeros((len(offsets) - 1, 23))
    lib.rs_diagnose_fields(len(offsets) - 1, off.ctypes.data_as(_i64p), _p(_c(w.pos)), _p(_c(w.alpha)),
                           _p(_c(w.sigma)), int(row_lo), int(row_hi), _p(out))
    return out
