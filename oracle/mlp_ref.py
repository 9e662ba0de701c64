"""FP64 numpy restatement of the far-field correction network (24-128-128-128-6,
GELU tanh form) for gradient checks.  TEST INFRASTRUCTURE ONLY.

The parameter vector uses the library's layout (include/pawan_gpu.h):
W1[32][128] (rows 24..31 zero), b1[128], W2[128][128], b2, W3[128][128], b3,
W4[128][8] (columns 6, 7 zero), b4[8].  Loss: mean squared error over the 6
outputs.  The model has no PAWAN counterpart; it is checked against this
restatement and against finite differences of it.
"""
from __future__ import annotations

import numpy as np

IN, INP, HID, OUT, OUTP = 24, 32, 128, 6, 8
OFF = {}
_o = 0
for name, size in (("W1", INP * HID), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("W3", HID * HID), ("b3", HID),
                   ("W4", HID * OUTP), ("b4", OUTP)):
    OFF[name] = (_o, size)
    _o += size
NUM_PARAMS = _o
SHAPES = {"W1": (INP, HID), "b1": (HID,), "W2": (HID, HID), "b2": (HID,), "W3": (HID, HID), "b3": (HID,),
          "W4": (HID, OUTP), "b4": (OUTP,)}
K0, K1 = np.sqrt(2.0 / np.pi), 0.044715


def unpack(p):
    return {k: np.asarray(p[o:o + s], np.float64).reshape(SHAPES[k]) for k, (o, s) in OFF.items()}


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * K0 * (1 + 3 * K1 * z * z)


def forward(p, x):
    P = unpack(p)
    X = np.zeros((x.shape[0], INP))
    X[:, :IN] = x
    Z1 = X @ P["W1"] + P["b1"]
    H1 = gelu(Z1)
    Z2 = H1 @ P["W2"] + P["b2"]
    H2 = gelu(Z2)
    Z3 = H2 @ P["W3"] + P["b3"]
    H3 = gelu(Z3)
    Y = H3 @ P["W4"] + P["b4"]
    return Y[:, :OUT], (X, Z1, H1, Z2, H2, Z3, H3, Y)


def loss_and_grad(p, x, t):
    P = unpack(p)
    y, (X, Z1, H1, Z2, H2, Z3, H3, Y) = forward(p, x)
    n = x.shape[0]
    d = y - t
    loss = float(np.sum(d * d) / (n * OUT))
    dY = np.zeros_like(Y)
    dY[:, :OUT] = 2 * d / (n * OUT)
    g = {}
    g["W4"] = H3.T @ dY
    g["b4"] = dY.sum(0)
    dZ3 = (dY @ P["W4"].T) * gelu_grad(Z3)
    g["W3"] = H2.T @ dZ3
    g["b3"] = dZ3.sum(0)
    dZ2 = (dZ3 @ P["W3"].T) * gelu_grad(Z2)
    g["W2"] = H1.T @ dZ2
    g["b2"] = dZ2.sum(0)
    dZ1 = (dZ2 @ P["W2"].T) * gelu_grad(Z1)
    g["W1"] = X.T @ dZ1
    g["b1"] = dZ1.sum(0)
    g["W4"][:, OUT:] = 0
    g["b4"][OUT:] = 0
    g["W1"][IN:, :] = 0
    flat = np.zeros(NUM_PARAMS)
    for k, (o, s) in OFF.items():
        flat[o:o + s] = g[k].ravel()
    return loss, flat


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights (numpy RNG; used by tests, not bit-identical to the library's init)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NUM_PARAMS)
    for k, (fi, fo) in (("W1", (IN, HID)), ("W2", (HID, HID)), ("W3", (HID, HID)), ("W4", (HID, OUT))):
        o, s = OFF[k]
        W = np.zeros(SHAPES[k])
        lim = np.sqrt(6.0 / (fi + fo))
        W[:fi, :fo] = rng.uniform(-lim, lim, (fi, fo))
        p[o:o + s] = W.ravel()
    return p
