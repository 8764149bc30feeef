"""Float64 restatement of the learned-proposal network -- TEST INFRASTRUCTURE
ONLY (the gradient check of the CUDA training kernels in csrc/mlp.cu).

48 -> 128 -> 128 -> 128 -> 40, SiLU between layers; outputs per component k:
mean m_k (3, normalised), concentration kappa_k = softplus(raw) + 1e-3,
weight logit.  Loss: mean over samples of -log sum_k pi_k C(kappa_k)
exp(kappa_k mu_k . x), C(kappa) = kappa / (4 pi sinh kappa).
"""

from __future__ import annotations

import math

import numpy as np

SHAPES = [(128, 48), (128, 128), (128, 128), (40, 128)]


def unpack(params):
    p = np.asarray(params, np.float64)
    out, off = [], 0
    for o, i in SHAPES:
        W = p[off:off + o * i].reshape(o, i)
        b = p[off + o * i:off + o * i + o]
        out.append((W, b))
        off += o * i + o
    return out


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s + z * s * (1.0 - s)


def forward(params, X):
    layers = unpack(params)
    a = np.asarray(X, np.float64)
    acts, zs = [a], []
    for l, (W, b) in enumerate(layers):
        z = a @ W.T + b
        zs.append(z)
        a = _silu(z) if l < 3 else z
        acts.append(a)
    return a, acts, zs


def nll_and_grad(Y, T):
    """Mean NLL and its gradient w.r.t. Y (both float64)."""
    B = Y.shape[0]
    y = Y.reshape(B, 8, 5)
    m = y[..., :3]
    nrm = np.linalg.norm(m, axis=-1) + 1e-12
    mu = m / nrm[..., None]
    kr = y[..., 3]
    kap = np.where(kr > 20, kr, np.log1p(np.exp(np.minimum(kr, 20)))) + 1e-3
    lg = y[..., 4]
    lse_l = lg.max(-1, keepdims=True) + np.log(np.exp(lg - lg.max(-1, keepdims=True)).sum(-1, keepdims=True))
    logpi = lg - lse_l
    dot = np.einsum("bkc,bc->bk", mu, T)
    logsinh = kap + np.log1p(-np.exp(-2 * kap)) - math.log(2)
    s = logpi + np.log(kap) - math.log(4 * math.pi) - logsinh + kap * dot
    lse = s.max(-1, keepdims=True) + np.log(np.exp(s - s.max(-1, keepdims=True)).sum(-1, keepdims=True))
    loss = -lse[:, 0]
    r = np.exp(s - lse)
    pi = np.exp(logpi)
    fk = np.where(kap < 1e-3, -kap / 3, 1 / kap - 1 / np.tanh(kap))
    g = np.zeros_like(y)
    g[..., 4] = pi - r
    g[..., 3] = -r * (fk + dot) / (1 + np.exp(-kr))
    c = -r * kap / nrm
    g[..., :3] = c[..., None] * (T[:, None, :] - dot[..., None] * mu)
    return loss.mean(), g.reshape(B, 40) / B


def grads(params, X, T):
    """Mean loss and the flat parameter gradient (layout W1 b1 ... W4 b4)."""
    layers = unpack(params)
    Y, acts, zs = forward(params, X)
    loss, dz = nll_and_grad(Y, np.asarray(T, np.float64))
    out = [None] * 4
    for l in range(3, -1, -1):
        W, _ = layers[l]
        gW = dz.T @ acts[l]
        gb = dz.sum(0)
        out[l] = (gW, gb)
        if l == 0:
            break
        dz = (dz @ W) * _dsilu(zs[l - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in out])
    return loss, flat
