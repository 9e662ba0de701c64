"""The far-field correction network: this library's BF16 tensor-core forward,
backward and Adam kernels against the FP64 numpy restatement (oracle/mlp_ref.py),
and what the trained network gains over the monopole+dipole far field."""
import numpy as np
import pytest

from oracle import mlp_ref as R
from oracle import oracle as O
from pawan_b200 import capi, cases


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = R.init_params(1)
    p[R.OFF["b1"][0]:R.OFF["b1"][0] + 128] = rng.normal(0, 0.1, 128)
    x = rng.normal(size=(7, R.IN))
    t = rng.normal(size=(7, R.OUT))
    _, g = R.loss_and_grad(p, x, t)
    for name in ("W1", "b1", "W2", "W3", "b3", "W4", "b4"):
        o, s = R.OFF[name]
        for k in rng.choice(s, 4, replace=False):
            i = o + k
            if name == "W1" and k // 128 >= R.IN or name in ("W4",) and k % 8 >= R.OUT or name == "b4" and k >= R.OUT:
                continue
            e = np.zeros_like(p)
            e[i] = 1e-6
            fd = (R.loss_and_grad(p + e, x, t)[0] - R.loss_and_grad(p - e, x, t)[0]) / 2e-6
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (name, k, fd, g[i])


@pytest.mark.gpu
def test_forward_matches_oracle(gpu):
    m = capi.Mlp(seed=3)
    p = m.params.astype(np.float64)
    x = np.random.default_rng(1).normal(size=(1000, R.IN)).astype(np.float32)
    y = m.forward(x)
    yr, _ = R.forward(p, x.astype(np.float64))
    assert np.abs(y - yr).max() <= 2e-2 * np.abs(yr).max()


@pytest.mark.gpu
def test_fused_inference_matches_forward(gpu):
    """The warp-level path the far field uses gives the training network's outputs."""
    m = capi.Mlp(seed=9)
    x = np.random.default_rng(6).normal(size=(1001, R.IN)).astype(np.float32)
    y = m.forward(x)
    yf = m.forward_fused(x)
    assert np.abs(yf - y).max() <= 1e-2 * np.abs(y).max()


@pytest.mark.gpu
def test_gradient_matches_oracle(gpu):
    """BF16 operands with FP32 accumulation against FP64: per-tensor relative
    error of the gradient below 5e-2."""
    m = capi.Mlp(seed=5)
    p = m.params.astype(np.float64)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(4096, R.IN)).astype(np.float32)
    t = rng.normal(size=(4096, R.OUT)).astype(np.float32)
    loss, g = m.gradient(x, t)
    lr_, gr = R.loss_and_grad(p, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lr_) <= 1e-2 * lr_
    for name, (o, s) in R.OFF.items():
        a, b = g[o:o + s].astype(np.float64), gr[o:o + s]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-9, name


@pytest.mark.gpu
def test_training_reduces_loss(gpu):
    rng = np.random.default_rng(4)
    x = rng.normal(size=(20000, R.IN)).astype(np.float32)
    A = rng.normal(size=(R.IN, R.OUT)) / np.sqrt(R.IN)
    t = np.tanh(x @ A).astype(np.float32)
    m = capi.Mlp(seed=7)
    m.set_dataset(x, t)
    hist = m.train(400, batch=2048, lr=2e-3, seed=1)
    assert np.all(np.isfinite(hist))
    assert hist[-20:].mean() < 0.1 * hist[:5].mean()


# Leaf size of the octree for the systems of 20k particles and more, in
# training and in evaluation alike: the network is trained on the cells of
# one leaf size and does not carry over to another.
LEAF = 256
# The network's test runs at four cube widths: there the dipole far field
# covers the cells nearest the near field, whose residual the network learns
WIDTHS = 4.0


def surrogate_rates(w, order, mlp=None):
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.surrogate_enable(order=order, use_mlp=1 if mlp is not None else 0, check_targets=0, leaf_size=LEAF,
                       near_widths=WIDTHS)
    if mlp is not None:
        c.surrogate_set_mlp(mlp)
    c.solve()
    v, a = c.rates(k)
    c.close()
    return v, a


def training_set(mlp, n_per_case=200_000):
    """Samples from the single-ring (5000), 1M-style Gaussian ring (200 stations)
    and uneven-ring workloads."""
    ws = [cases.ring_stations(), cases.ring_gaussian(stations=200, seed=1)]
    ws += cases.uneven_rings(count=4, nmin=20_000, nmax=200_000, seed=2)
    for i, w in enumerate(ws):
        c = capi.Context(precision=capi.FP32C, nu=1e-4)
        k = c.add_wake(w.n)
        c.set_particles(k, w)
        # the 5000-particle ring has far cells only with small leaves; the
        # features are scale-free, so samples of any leaf size mix
        c.surrogate_enable(order=1, check_targets=0, leaf_size=32 if w.n < 20_000 else LEAF, near_widths=WIDTHS)
        c.solve()
        mlp.add_samples(c, n_per_case, seed=i)
        c.close()


@pytest.mark.gpu
@pytest.mark.slow
def test_trained_network_improves_dipole_far_field(gpu):
    mlp = capi.Mlp(seed=11)
    training_set(mlp)
    x, t = mlp.dataset(10_000)
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(t)) and np.abs(t).max() > 0
    hist = mlp.train(3000, batch=16384, lr=1e-3, seed=3)
    assert hist[-50:].mean() < 0.5 * hist[:20].mean()
    w = cases.leapfrog_rings(n_total=200_000)
    c = capi.Context(precision=capi.FP32C, nu=1e-4)
    k = c.add_wake(w.n)
    c.set_particles(k, w)
    c.solve()
    vd, ad = c.rates(k)
    c.close()
    e1 = O.rel_err(surrogate_rates(w, 1)[0], vd)
    em = O.rel_err(surrogate_rates(w, 1, mlp)[0], vd)
    e2 = O.rel_err(surrogate_rates(w, 2)[0], vd)
    print(f"far-field velocity error: dipole {e1:.3e}, dipole + network {em:.3e}, quadrupole {e2:.3e}")
    assert em < e1
