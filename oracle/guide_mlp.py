"""Test infrastructure (CPU oracle): the learned guide's MLP, mixture head and
gradients in numpy, for checking the tensor-core kernels of
cenote_b200/csrc/guide.cu.

`forward`/`backward` emulate the kernels' precision: BF16 inputs, weights
and activations between layers, FP32 accumulation and biases, BF16 dZ at
each layer's input to the MMAs. `mixture_*` restate the vMF mixture head of
cenote_b200/csrc/guide.h in float64. `loss_and_grad64` is the same model in
float64 without rounding, for finite-difference checks of the analytic
gradient. The objective is the KL estimator of neural importance sampling
(Müller et al. 2019): mean_s -c_s log q(w_s).
"""
from __future__ import annotations

import numpy as np

IN, HIDDEN, LOBES = 96, 64, 8
OUT = 5 * LOBES
SIZES = [(HIDDEN, IN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUT, HIDDEN)]


def unpack(p):
    """Weights [out][in] and biases from the flat FP32 parameter vector."""
    out, o = [], 0
    for n, k in SIZES:
        w = p[o:o + n * k].reshape(n, k)
        o += n * k
        b = p[o:o + n]
        o += n
        out.append((w, b))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([w.reshape(-1), b]) for w, b in layers]).astype(np.float32)


def bf16(x):
    """Round float32 values to BF16 (nearest even) and back."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def forward(params, x):
    """Outputs and the saved BF16 activations, as the kernels compute them."""
    acts = [bf16(x)]
    a = acts[0]
    for l, (w, b) in enumerate(unpack(params)):
        z = a.astype(np.float32) @ bf16(w).T.astype(np.float32) + b
        if l < 3:
            a = bf16(np.maximum(z, 0.0))
            acts.append(a)
        else:
            return z.astype(np.float32), acts


def lobes(o):
    o = np.asarray(o, np.float64).reshape(-1, LOBES, 5)
    r = o[..., :3]
    n = np.sqrt((r ** 2).sum(-1) + 1e-12)
    mu = r / n[..., None]
    x = np.clip(o[..., 3], -20, 20)
    kappa = 0.01 + np.log1p(np.exp(x))
    logits = o[..., 4]
    w = np.exp(logits - logits.max(-1, keepdims=True))
    w /= w.sum(-1, keepdims=True)
    return mu, kappa, w, n, x


def vmf(kappa, cosw):
    return kappa / (2 * np.pi * (1 - np.exp(-2 * kappa))) * np.exp(kappa * (cosw - 1))


def mixture_pdf(o, dirs):
    """q(w) for outputs (n, 40) and unit directions (n, 3)."""
    mu, kappa, w, _, _ = lobes(o)
    cosw = (mu * np.asarray(dirs, np.float64)[:, None, :]).sum(-1)
    return (w * vmf(kappa, cosw)).sum(-1)


def mixture_grad(o, dirs, c):
    """d(-c log q(w))/d(outputs), float64, (n, 40); and log q."""
    mu, kappa, w, n, x = lobes(o)
    d = np.asarray(dirs, np.float64)
    cosw = (mu * d[:, None, :]).sum(-1)
    v = vmf(kappa, cosw)
    q = np.maximum((w * v).sum(-1), 1e-20)
    dq = -np.asarray(c, np.float64) / q
    g = np.zeros((len(q), LOBES, 5))
    g[..., 4] = dq[:, None] * w * (v - q[:, None])
    e2 = np.exp(-2 * kappa)
    dv_dk = v * (1 / kappa - 2 * e2 / (1 - e2) + (cosw - 1))
    g[..., 3] = dq[:, None] * w * dv_dk / (1 + np.exp(-x))
    s = dq[:, None] * w * v * kappa / n
    g[..., :3] = s[..., None] * (d[:, None, :] - cosw[..., None] * mu)
    return g.reshape(-1, OUT), np.log(q)


def backward(params, acts, dout):
    """dL/dparams from the kernels' saved activations and dZ4 = dout (FP32)."""
    layers = unpack(params)
    grads = [None] * 4
    dz = bf16(dout)
    for l in range(3, -1, -1):
        w, _ = layers[l]
        a_in = acts[l].astype(np.float64)
        grads[l] = (dz.astype(np.float64).T @ a_in, dz.astype(np.float64).sum(0))
        if l > 0:
            da = dz.astype(np.float32) @ bf16(w).astype(np.float32)
            dz = bf16(np.where(acts[l] > 0, da, 0.0))
    return np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])


def loss_and_grad64(params, x, dirs, c):
    """The same model in float64, no rounding: (loss, gradient)."""
    layers = [(w.astype(np.float64), b.astype(np.float64)) for w, b in unpack(np.asarray(params, np.float64))]
    a = [np.asarray(x, np.float64)]
    for l, (w, b) in enumerate(layers):
        z = a[-1] @ w.T + b
        a.append(np.maximum(z, 0) if l < 3 else z)
    n = len(x)
    g, logq = mixture_grad(a[-1], dirs, np.asarray(c) / n)
    loss = float(-(np.asarray(c) / n * logq).sum())
    grads = [None] * 4
    dz = g
    for l in range(3, -1, -1):
        w, _ = layers[l]
        grads[l] = (dz.T @ a[l], dz.sum(0))
        if l > 0:
            dz = (dz @ w) * (a[l] > 0)
    return loss, np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])
