"""The learned guide's MLP: tensor-core forward/backward against the numpy oracle.

CPU: the oracle's analytic gradient against central finite differences in
float64, and the vMF mixture's normalisation. GPU: the tcgen05 kernels'
outputs and gradients against the oracle's emulation of their precision
(BF16 operands, FP32 accumulation), an Adam step, and a training run that
fits a known directional distribution.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import guide_mlp as M


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    layers = []
    for n, k in M.SIZES:
        a = np.sqrt(6.0 / k)
        layers.append((rng.uniform(-a, a, (n, k)).astype(np.float32), rng.normal(0, 0.05, n).astype(np.float32)))
    return M.pack(layers)


def batch(n, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, M.IN)).astype(np.float32)
    x[:, 81:] = 0.0
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    c = rng.exponential(1.0, n)
    return x, d.astype(np.float32), c.astype(np.float32)


# ---- oracle self-checks --------------------------------------------------------------


def test_oracle_gradient_matches_finite_differences():
    p = init_params().astype(np.float64)
    x, d, c = batch(12)
    loss, g = M.loss_and_grad64(p, x, d, c)
    rng = np.random.default_rng(4)
    idx = rng.choice(len(p), 60, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad64(pp, x, d, c)[0] - M.loss_and_grad64(pm, x, d, c)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_mixture_is_a_density():
    rng = np.random.default_rng(7)
    o = rng.normal(0, 2, (4, M.OUT))
    # Fibonacci sphere quadrature.
    n = 200000
    k = np.arange(n) + 0.5
    z = 1 - 2 * k / n
    phi = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], -1)
    for row in o:
        q = M.mixture_pdf(np.repeat(row[None], n, 0), dirs)
        assert abs(q.mean() * 4 * np.pi - 1.0) < 2e-3


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -2.5], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125) and r[4] == -2.5


# ---- the tensor-core kernels -----------------------------------------------------------


@pytest.fixture(scope="module")
def net(ctx):
    from cenote_b200 import Guide

    g = Guide(ctx, seed=3)
    yield g
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 1000, 20000])
def test_gpu_forward_matches_oracle(net, n):
    p = init_params(5)
    net.set_params(p)
    x, _, _ = batch(n, seed=n)
    got = net.forward(x)
    ref, _ = M.forward(p, x)
    scale = np.abs(ref).max() + 1e-6
    err = np.abs(got - ref)
    assert err.max() <= 2e-3 * scale, (err.max(), scale)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [100, 4096, 65536])
def test_gpu_gradient_matches_oracle(net, n):
    p = init_params(6)
    net.set_params(p)
    x, d, c = batch(n, seed=11)
    loss, g = net.train_step(x, d, c, lr=0.0, grads=True)
    out, acts = M.forward(p, x)
    dout, logq = M.mixture_grad(out, d, c / n)
    ref_loss = float(-(c / n * logq).sum())
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss) + 1e-4
    ref = M.backward(p, acts, dout.astype(np.float32))
    off = 0
    for nk in M.SIZES:
        for size in (nk[0] * nk[1], nk[0]):
            a, b = g[off:off + size], ref[off:off + size]
            rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
            assert rel < 2e-2, (off, size, rel)
            off += size


@pytest.mark.gpu
def test_gpu_adam_step(net):
    p = init_params(8)
    net.set_params(p)
    x, d, c = batch(2048, seed=3)
    _, g = net.train_step(x, d, c, lr=0.0, grads=True)
    net.set_params(p)
    net.train_step(x, d, c, lr=1e-2)
    after = net.params()
    # First Adam step: m = 0.1 g, v = 0.001 g^2, bias-corrected -> p - lr * g / (|g| + eps).
    expect = p - 1e-2 * g / (np.sqrt(g * g) + 1e-8)
    assert np.allclose(after, expect, atol=2e-5)


@pytest.mark.gpu
def test_gpu_training_fits_a_directional_distribution(net):
    """Directions drawn from a vMF around an axis that depends on the first
    input feature; training must concentrate q there."""
    rng = np.random.default_rng(12)
    net.set_params(init_params(9))

    def sample(n):
        x = np.zeros((n, M.IN), np.float32)
        s = rng.uniform(-1, 1, n)
        x[:, 0] = s
        x[:, 1] = 1.0
        axis = np.stack([np.sin(s * 1.2), np.zeros(n), np.cos(s * 1.2)], -1)
        # vMF(kappa = 20) around axis: sample cos theta exactly.
        u = rng.random(n)
        kappa = 20.0
        cos = 1 + np.log(u + (1 - u) * np.exp(-2 * kappa)) / kappa
        phi = rng.uniform(0, 2 * np.pi, n)
        sin = np.sqrt(np.maximum(0, 1 - cos * cos))
        t = np.cross(axis, [0.0, 1.0, 0.0])
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        b = np.cross(axis, t)
        d = cos[:, None] * axis + sin[:, None] * (np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * b)
        return x, d.astype(np.float32), axis

    x0, d0, axis0 = sample(4096)
    before = np.log(M.mixture_pdf(net.forward(x0), axis0)).mean()
    losses = []
    for _ in range(300):
        x, d, _ = sample(8192)
        losses.append(net.train_step(x, d, np.ones(len(x), np.float32), lr=5e-3))
    after = np.log(M.mixture_pdf(net.forward(x0), axis0)).mean()
    assert np.mean(losses[-20:]) < np.mean(losses[:20]) - 1.0
    assert after > before + 2.0  # the density at the axis rose by more than e^2
