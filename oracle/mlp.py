"""Test infrastructure: float64 NumPy restatement of the learned closure's network and its
training loss -- the checker for the library's hand-written CUDA forward/backward kernels.
It is never imported by the product.

Layout (as zsmpm_closure_state.params): W1[64][6] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
W4[6][64] b4[6]; SiLU on the three hidden layers; loss = mean over samples and outputs of the
squared error of normalised outputs, inputs normalised as (x - mean) * inv_std, targets as
y / out_scale.
"""
from __future__ import annotations

import numpy as np

SIZES = [(64, 6), (64, 64), (64, 64), (6, 64)]
N_PARAMS = sum(o * i + o for o, i in SIZES)


def inputs(model, raw, kappa, hardening=0.0):
    """Raw feature rows [n, 6] -> (network inputs, sD, sT, off) with D = sD o[:3] and
    tau = off + sT o[3:].  Drucker-Prager (model 1): eps = l - c, s = |(eps, logJp)|, inputs
    (eps / s, logJp / s, friction, tr / s), sD = s, sT = kappa s, off = kappa c (the return map
    is positively homogeneous of degree one in (eps, logJp)).  Snow: u = (l - mid) / half in the
    clamp box [log(1 - theta_c), log(1 + theta_s)], inputs (u, theta_c, theta_s, log Jp),
    sD = half, sT = kappa exp(xi (1 - Jp)), off = 0."""
    raw = np.asarray(raw, np.float64)
    if model == 1:
        eps = raw[:, :3] - raw[:, 4:5]
        s = np.sqrt(np.sum(eps * eps, 1) + raw[:, 5] ** 2) + 1e-12
        d = eps / s[:, None]
        pj = raw[:, 5] / s
        x = np.stack([d[:, 0], d[:, 1], d[:, 2], pj, raw[:, 3], d.sum(1) + pj], 1)
        return x, s, kappa * s, kappa * raw[:, 4]
    lo, hi = np.log1p(-raw[:, 3]), np.log1p(raw[:, 4])
    mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    x = np.concatenate([(raw[:, :3] - mid[:, None]) / half[:, None], raw[:, 3:]], 1)
    return x, half, kappa * np.exp(hardening * (1 - np.exp(raw[:, 5]))), np.zeros(len(raw))


def net_targets(model, raw, y, kappa, hardening=0.0):
    """(D, tau) rows -> the network's targets."""
    _, sD, sT, off = inputs(model, raw, kappa, hardening)
    y = np.asarray(y, np.float64)
    return np.concatenate([y[:, :3] / sD[:, None], (y[:, 3:] - off[:, None]) / sT[:, None]], 1)


def from_net(model, raw, o, kappa, hardening=0.0):
    """The network's outputs -> (D, tau); the inverse of net_targets."""
    _, sD, sT, off = inputs(model, raw, kappa, hardening)
    o = np.asarray(o, np.float64)
    return np.concatenate([o[:, :3] * sD[:, None], off[:, None] + sT[:, None] * o[:, 3:]], 1)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, off = [], 0
    for o, i in SIZES:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, xn):
    """xn: normalised inputs [n,6] -> outputs [n,6] (normalised units)."""
    a = np.asarray(xn, np.float64)
    for k, (W, b) in enumerate(unpack(p)):
        z = a @ W.T + b
        a = silu(z) if k < 3 else z
    return a


def loss_and_grad(p, xn, yn):
    """Mean squared error and its gradient with respect to the flat parameter vector."""
    layers = unpack(p)
    acts, zs = [np.asarray(xn, np.float64)], []
    a = acts[0]
    for k, (W, b) in enumerate(layers):
        z = a @ W.T + b
        zs.append(z)
        a = silu(z) if k < 3 else z
        acts.append(a)
    n = len(xn)
    err = a - yn
    loss = float(np.sum(err * err) / (n * 6))
    d = 2.0 * err / (n * 6)
    grads = []
    for k in range(3, -1, -1):
        W, _ = layers[k]
        if k < 3:
            d = d * silu_grad(zs[k])
        grads.append((d.T @ acts[k], d.sum(0)))
        d = d @ W
    flat = []
    for gW, gb in reversed(grads):
        flat.append(gW.ravel())
        flat.append(gb)
    return loss, np.concatenate(flat)
