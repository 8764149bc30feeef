"""Learned von Mises-Fisher mixture proposal for the probabilistic getter.

A 48 -> 128 -> 128 -> 128 -> 40 SiLU MLP maps the 45 interpolated SH
coefficients at a position plus the incoming direction to an 8-component vMF
mixture over the next direction.  It is trained on the steps the plain
probabilistic tracker takes, with the library's own CUDA kernels (forward
GEMMs, SiLU, the mixture negative log-likelihood and its gradient, the
backward GEMMs, Adam; see csrc/mlp.cu); torch only holds the device memory and
runs the training loop.

Use as a proposal: exact rejection sampling of the probabilistic getter's
target (the thresholded, cone-filtered PMF over the sphere vertices) with the
mixture -- restricted to the cone and mixed with 30 % of the uniform-cone
proposal (a defensive mixture, which bounds p / q where the network's tails
are too thin) -- accepts with probability 1 / max_v p(v) / q(v), so the
sampled distribution is the target's whatever the network; the network only
changes how many draws a step needs.  ``acceptance`` measures that rate against
the uniform-cone proposal the method would use without the network.  Bounding
max p/q needs the whole PMF at the position, so on this getter the proposal
does not remove the 724-vertex gather that bounds the plain kernel.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

N_IN, N_HID, N_OUT, N_COMP = 48, 128, 40, 8
SHAPES = [(N_HID, N_IN), (N_HID, N_HID), (N_HID, N_HID), (N_OUT, N_HID)]


def _vp(t):
    return C.c_void_p(t.data_ptr())


class VmfProposalNet:
    """Parameters (flat FP32 device tensor, layout W1 b1 W2 b2 W3 b3 W4 b4) and Adam state."""

    def __init__(self, device: int = 0, seed: int = 0):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.lib = _lib.load()
        n = self.lib.csl_mlp_param_count()
        rng = np.random.default_rng(seed)
        p = np.zeros(n, dtype=np.float32)
        off = 0
        self.views = []
        for (o, i) in SHAPES:
            w = rng.uniform(-1, 1, (o, i)) * math.sqrt(6.0 / (i + o))
            p[off:off + o * i] = w.ravel()
            self.views.append((off, o, i))
            off += o * i + o
        assert off == n
        self.params = torch.from_numpy(p).to(self.dev)
        self.grad = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.feat_mean = np.zeros(N_IN, np.float32)
        self.feat_std = np.ones(N_IN, np.float32)

    def _w(self, l):
        off, o, i = self.views[l]
        return self.params[off:off + o * i], self.params[off + o * i:off + o * i + o]

    def _g(self, l):
        off, o, i = self.views[l]
        return self.grad[off:off + o * i], self.grad[off + o * i:off + o * i + o]

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(f"MLP kernel failed ({rc})")

    def forward(self, X):
        """X [B, 48] device -> Y [B, 40]; keeps the activations for backward."""
        torch = self.torch
        B = X.shape[0]
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        self.cache = [X]
        self.zs = []
        a = X
        for l, (o, i) in enumerate(SHAPES):
            W, b = self._w(l)
            z = torch.empty((B, o), dtype=torch.float32, device=self.dev)
            self._chk(self.lib.csl_mlp_gemm(0, 1, B, o, i, _vp(a), i, _vp(W), i, _vp(z), o, 0.0, st))
            out = torch.empty_like(z)
            self._chk(self.lib.csl_mlp_bias_act(_vp(z), _vp(b), _vp(out), B, o, 1 if l < 3 else 0, st))
            self.zs.append(z)
            self.cache.append(out)
            a = out
        return a

    def backward(self, dY):
        """Gradients of all parameters from dY [B, 40] into self.grad."""
        torch = self.torch
        B = dY.shape[0]
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        dz = dY
        for l in range(3, -1, -1):
            o, i = SHAPES[l]
            W, _ = self._w(l)
            gW, gb = self._g(l)
            a_prev = self.cache[l]
            self._chk(self.lib.csl_mlp_gemm(1, 0, o, i, B, _vp(dz), o, _vp(a_prev), i, _vp(gW), i, 0.0, st))
            self._chk(self.lib.csl_mlp_colsum(_vp(dz), B, o, _vp(gb), st))
            if l == 0:
                break
            da = torch.empty((B, i), dtype=torch.float32, device=self.dev)
            self._chk(self.lib.csl_mlp_gemm(0, 0, B, i, o, _vp(dz), o, _vp(W), i, _vp(da), i, 0.0, st))
            dzp = torch.empty_like(da)
            self._chk(self.lib.csl_mlp_act_bwd(_vp(self.zs[l - 1]), _vp(da), _vp(dzp), B * i, st))
            dz = dzp

    def loss_and_grad(self, X, T):
        """Mean mixture NLL of unit targets T [B, 3]; fills self.grad."""
        torch = self.torch
        B = X.shape[0]
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        Y = self.forward(X)
        loss = torch.empty(B, dtype=torch.float32, device=self.dev)
        dY = torch.empty_like(Y)
        self._chk(self.lib.csl_mlp_vmf_nll(_vp(Y), _vp(T), B, 1.0 / B, _vp(loss), _vp(dY), st))
        self.backward(dY)
        return loss

    def train_step(self, X, T, lr=1e-3):
        torch = self.torch
        loss = self.loss_and_grad(X, T)
        self.step += 1
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        self._chk(self.lib.csl_mlp_adam(_vp(self.params), _vp(self.grad), _vp(self.m), _vp(self.v),
                                        self.params.numel(), lr, 0.9, 0.999, 1e-8, self.step, st))
        return loss

    def infer(self, X, return_ms=False):
        """Fused inference kernel (weights in shared memory): X [B, 48] -> Y [B, 40]."""
        torch = self.torch
        Y = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device=self.dev)
        ms = np.zeros(1, np.float32)
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        self._chk(self.lib.csl_mlp_infer(_vp(self.params), _vp(X), X.shape[0], _vp(Y), _lib.fptr(ms), st))
        return (Y, float(ms[0])) if return_ms else Y

    def features(self, sh, din):
        """Standardised network inputs from SH coefficients [B, 45] and directions [B, 3]."""
        f = np.concatenate([np.asarray(sh, np.float32), np.asarray(din, np.float32)], axis=1)
        return (f - self.feat_mean) / self.feat_std


def mixture(Y):
    """Network outputs [B, 40] -> (mu [B, 8, 3], kappa [B, 8], log_pi [B, 8]) in float64."""
    y = np.asarray(Y, np.float64).reshape(-1, N_COMP, 5)
    m = y[..., :3]
    mu = m / (np.linalg.norm(m, axis=-1, keepdims=True) + 1e-12)
    kr = y[..., 3]
    kappa = np.where(kr > 20, kr, np.log1p(np.exp(np.minimum(kr, 20)))) + 1e-3
    lg = y[..., 4]
    log_pi = lg - (np.log(np.exp(lg - lg.max(-1, keepdims=True)).sum(-1, keepdims=True)) + lg.max(-1, keepdims=True))
    return mu, kappa, log_pi


def mixture_logpdf(mu, kappa, log_pi, x):
    """log density of unit vectors x [B, n, 3] under each row's mixture -> [B, n]."""
    logsinh = kappa + np.log1p(-np.exp(-2 * kappa)) - math.log(2)
    logc = np.log(kappa) - math.log(4 * math.pi) - logsinh            # [B, 8]
    dots = np.einsum("bkc,bnc->bnk", mu, x)                          # [B, n, 8]
    s = log_pi[:, None, :] + logc[:, None, :] + kappa[:, None, :] * dots
    mx = s.max(-1, keepdims=True)
    return (mx + np.log(np.exp(s - mx).sum(-1, keepdims=True)))[..., 0]


def trilinear(vol, pts):
    """Trilinear interpolation of vol [X, Y, Z, C] at pts [n, 3] (clamped corners) -> [n, C] float64."""
    X, Y, Z = vol.shape[:3]
    p = np.asarray(pts, np.float64)
    fl = np.floor(p)
    w1 = p - fl
    lo = np.clip(fl, 0, np.array([X - 1, Y - 1, Z - 1])).astype(np.int64)
    hi = np.minimum(lo + 1, np.array([X - 1, Y - 1, Z - 1]))
    out = 0.0
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                cx = (lo if i == 0 else hi)[:, 0]
                cy = (lo if j == 0 else hi)[:, 1]
                cz = (lo if k == 0 else hi)[:, 2]
                w = (w1[:, 0] if i else 1 - w1[:, 0]) * (w1[:, 1] if j else 1 - w1[:, 1]) * \
                    (w1[:, 2] if k else 1 - w1[:, 2])
                out = out + w[:, None] * vol[cx, cy, cz].astype(np.float64)
    return out


def steps_from_tracks(lengths, seed_ids, points, seeds):
    """(position, incoming direction, chosen direction) of every step of the
    tracked streamlines, in the order the tracker took them (both halves run
    outward from the seed)."""
    off = np.concatenate([[0], np.cumsum(lengths)])
    pos, din, dout = [], [], []
    for i in range(len(lengths)):
        s = points[off[i]:off[i + 1]].astype(np.float64)
        hit = np.nonzero(np.all(points[off[i]:off[i + 1]] == seeds[seed_ids[i]], axis=1))[0]
        if len(hit) == 0 or len(s) < 3:
            continue
        k = int(hit[0])
        for half in (s[k:], s[k::-1]):
            if len(half) < 3:
                continue
            d = np.diff(half, axis=0)
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            pos.append(half[1:-1])
            din.append(d[:-1])
            dout.append(d[1:])
    if not pos:
        return np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3))
    return np.concatenate(pos), np.concatenate(din), np.concatenate(dout)


def target_pmf(pmf_vol, verts, pts, din, cos_max, pmf_thr=0.05):
    """The probabilistic getter's target at each state: interpolated PMF,
    5 % threshold, cone |v . d| >= cos(max_angle); directions flipped into the
    incoming hemisphere.  -> (p [B, V] normalised, x [B, V, 3], cone mask)."""
    pm = np.maximum(trilinear(pmf_vol, pts), 0.0)
    pm[pm < pmf_thr * pm.max(axis=1, keepdims=True)] = 0.0
    dots = np.asarray(din, np.float64) @ np.asarray(verts, np.float64).T
    cone = np.abs(dots) >= cos_max
    p = pm * cone
    tot = p.sum(axis=1, keepdims=True)
    p = np.where(tot > 0, p / np.where(tot > 0, tot, 1), 0)
    x = np.sign(dots)[..., None] * np.asarray(verts, np.float64)[None]
    return p, x, cone


DEFENSIVE = 0.3  # weight of the uniform-cone component in the proposal


def acceptance(p, x, cone, mu, kappa, log_pi, eps=DEFENSIVE):
    """Exact-rejection acceptance rates per state: the learned proposal (the
    mixture restricted to the cone vertices, mixed with weight ``eps`` of the
    uniform-cone proposal so that its tails never fall below eps / N_cone --
    a defensive mixture; eps = 0 is the bare network) and the uniform-cone
    proposal alone."""
    lq = mixture_logpdf(mu, kappa, log_pi, x)
    lq = np.where(cone, lq, -np.inf)
    lq = lq - lq.max(axis=1, keepdims=True)
    q = np.exp(lq)
    q = q / q.sum(axis=1, keepdims=True)
    q = (1.0 - eps) * q + eps * cone / cone.sum(axis=1, keepdims=True)
    r = np.divide(p, q, out=np.zeros_like(p), where=p > 0)
    acc_l = 1.0 / r.max(axis=1)
    ncone = cone.sum(axis=1)
    acc_u = 1.0 / (p.max(axis=1) * ncone)
    return acc_l, acc_u, q
