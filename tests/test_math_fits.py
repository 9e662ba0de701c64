"""The FP32 pair kernel's own approximations, checked on the CPU in FP32
emulation against SciPy (CPU only).

* the erfcx fit used for 1 <= u < 50 (erf(y) = 1 - e^{-y^2} z P(t));
* the small-u series S(u), T(u) against the closed form in FP64;
* the far-field limit (q = 1/(4 pi rho^3), F = -3 q / rho^2, zeta = 0) at u >= 50.
"""
import math
import re
from pathlib import Path

import numpy as np
from scipy.special import erf

HDR = (Path(__file__).resolve().parents[1] / "pawan_b200" / "csrc" / "pair_math.cuh").read_text()


def consts(prefix):
    vals = {}
    for name, val in re.findall(r"#define (PGPU_%s\d+) ([-+0-9.e]+)f?" % prefix, HDR):
        vals[int(name[len("PGPU_") + len(prefix):])] = float(val.rstrip("f"))
    return [vals[k] for k in sorted(vals)]


def cfloat(name):
    return float(re.search(r"%s = ([-+0-9.e]+)f" % name, HDR).group(1))


def kernel_closed(u):
    """4 pi q sigma^3 and 4 pi F sigma^5 from the closed form (gaussian.h:47-60), FP64."""
    x = np.sqrt(u)
    k1 = math.sqrt(2 / math.pi)
    z = k1 * np.exp(-u / 2)
    q = (erf(x / math.sqrt(2)) / x - k1 * np.exp(-u / 2)) / u
    F = (z - 3 * q) / u
    return q, F


def test_erfcx_fit_fp32():
    E = np.array(consts("E"), dtype=np.float32)
    a, b = np.float32(cfloat("kErfcxA")), np.float32(cfloat("kErfcxB"))
    y = np.linspace(1 / math.sqrt(2), 5.0, 200001)
    z = (1.0 / y).astype(np.float32)
    t = (a * z + b).astype(np.float32)
    P = np.full_like(t, E[-1])
    for c in E[-2::-1]:
        P = (P * t + c).astype(np.float32)
    ey = np.exp(-y * y).astype(np.float32)
    approx = (np.float32(1) - ey * z * P).astype(np.float32)
    err = np.abs(approx.astype(np.float64) - erf(y))
    assert err.max() < 1.2e-7, err.max()


def test_series_matches_closed_form():
    S = consts("S")
    T = consts("T")
    for u in (1e-3, 0.1, 0.5, 0.99):
        Sv = sum(c * u ** k for k, c in enumerate(S))
        Tv = sum(c * u ** k for k, c in enumerate(T))
        q, F = kernel_closed(u)
        k1 = math.sqrt(2 / math.pi)
        assert abs(k1 * Sv - q) < 1e-9 * abs(q)
        assert abs(-k1 * Tv - F) < 1e-7 * abs(F)


def test_far_limit_error_bound():
    for u in (50.0, 80.0, 400.0):
        q, F = kernel_closed(u)
        x = math.sqrt(u)
        assert abs(1 / x ** 3 - q) < 1e-9 * q
        assert abs(-3 / x ** 5 - F) < 2e-9 * abs(F)
        assert math.exp(-u / 2) < 1.4e-11


def test_fp64_far_limit_is_exact_to_double_rounding():
    """FP64 kernels take q' = r^-3, F' = -3 r^-5 for u = rho^2 / sigma^2 >= 100:
    the closed form (gaussian.h:47-60) equals that limit to a few units of
    double rounding there (the erfc and e^{-u/2} terms are below 1e-21 of
    them; what remains is the rounding of the two ways of evaluating)."""
    import math
    for u in np.linspace(100.0, 400.0, 200):
        rb = math.sqrt(u)  # rho / sigma, sigma = 1
        zeta = math.exp(-0.5 * u) / (2 * math.pi) ** 1.5
        phi = math.erf(rb / math.sqrt(2)) / (4 * math.pi)
        q = (phi / rb - zeta) / rb ** 2
        F = (zeta - 3 * q) / rb ** 2
        q_far = 1 / (4 * math.pi * rb ** 3)
        F_far = -3 * q_far / rb ** 2
        assert abs(q - q_far) <= 1e-15 * q_far
        assert abs(F - F_far) <= 1e-15 * abs(F_far)
