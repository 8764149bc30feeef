"""Learned vMF-mixture proposal: the CUDA training kernels against the float64
restatement (oracle/mlp_ref.py), the fused inference kernel against the
training forward, and what a briefly trained network gains over the proposal
without it.

Bars: per parameter tensor, relative L2 error of the kernel gradient < 1e-4;
loss within 1e-5 relative; inference = training forward within 1e-4 of the
output scale.  Trained on the plain tracker's steps on one phantom for 400
Adam steps: held-out NLL at least 1.0 nat below the uniform-sphere value
log(4 pi) and below the uniform-cone value, and mean exact-rejection
acceptance of the learned proposal (defensive mixture, 30 % uniform cone) at
least 1.2x the uniform-cone proposal's (the sampled distribution is the target's in both
cases: the check compares turning angles of the two samplers, KS p > 1e-3).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gradients_match_float64_oracle():
    import torch

    from gpustreamlines_b200.learned import VmfProposalNet
    from oracle import mlp_ref

    net = VmfProposalNet(seed=3)
    rng = np.random.default_rng(0)
    B = 96
    X = rng.normal(size=(B, 48)).astype(np.float32)
    T = rng.normal(size=(B, 3))
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    T = T.astype(np.float32)
    loss = net.loss_and_grad(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    torch.cuda.synchronize()
    ref_loss, ref_g = mlp_ref.grads(net.params.cpu().numpy(), X, T)
    assert abs(float(loss.mean()) - ref_loss) <= 1e-5 * abs(ref_loss) + 1e-6
    g = net.grad.cpu().numpy().astype(np.float64)
    off = 0
    for o, i in mlp_ref.SHAPES:
        for n in (o * i, o):
            a, b = g[off:off + n], ref_g[off:off + n]
            assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-7
            off += n


def test_inference_kernel_matches_training_forward():
    import torch

    from gpustreamlines_b200.learned import VmfProposalNet

    net = VmfProposalNet(seed=4)
    X = torch.randn(1000, 48, device="cuda")
    y0 = net.forward(X)
    y1 = net.infer(X)
    torch.cuda.synchronize()
    assert float((y0 - y1).abs().max()) <= 1e-4 * float(y0.abs().max())


def test_training_gains_over_uniform_proposal():
    import torch
    from scipy.stats import ks_2samp

    from gpustreamlines_b200 import learned
    from oracle import cases
    from test_gpu_parity import _handle

    inp = cases.inputs("prob_s")
    ph = inp["phantom"]
    seeds = cases.seeds("prob_s", 3000, seed=31)
    h = _handle("prob_s")
    h.propagate(seeds)
    L, S, P = h.fetch()
    h.close()
    pos, din, dout = learned.steps_from_tracks(L, S, P, seeds)
    assert len(pos) > 20000
    sh = learned.trilinear(ph.sh_coef, pos)
    net = learned.VmfProposalNet(seed=1)
    f = np.concatenate([sh, din], axis=1)
    net.feat_mean = f.mean(0).astype(np.float32)
    net.feat_std = (f.std(0) + 1e-6).astype(np.float32)
    X = torch.from_numpy(net.features(sh, din)).cuda()
    T = torch.from_numpy(dout.astype(np.float32)).cuda()
    n = len(pos)
    rng = np.random.default_rng(2)
    perm = rng.permutation(n)
    test, train = perm[:2000], perm[2000:]
    for it in range(400):
        idx = torch.from_numpy(train[rng.integers(0, len(train), 1024)]).cuda()
        net.train_step(X[idx], T[idx], lr=2e-3)
    ti = torch.from_numpy(test).cuda()
    nll = float(net.loss_and_grad(X[ti], T[ti]).mean())
    cos_max = math.cos(math.radians(inp["case"]["max_angle"]))
    assert nll < math.log(4 * math.pi) - 1.0
    assert nll < math.log(2 * math.pi * (1 - cos_max))

    Y = net.infer(X[ti]).cpu().numpy()
    mu, kappa, log_pi = learned.mixture(Y)
    p, x, cone = learned.target_pmf(inp["dataf"], inp["vertices"], pos[test], din[test], cos_max)
    ok = p.sum(axis=1) > 0
    acc_l, acc_u, q = learned.acceptance(p[ok], x[ok], cone[ok], mu[ok], kappa[ok], log_pi[ok])
    assert acc_l.mean() > 1.2 * acc_u.mean()
    # exact rejection sampling leaves the target unchanged: turning angles of
    # inverse-CDF draws and of learned-proposal rejection draws agree
    r = np.random.default_rng(5)
    a_exact, a_rej = [], []
    dd = din[test][ok]
    for b in range(min(1500, len(p[ok]))):
        pb, qb, xb = p[ok][b], q[b], x[ok][b]
        v = r.choice(len(pb), p=pb)
        a_exact.append(float(np.dot(xb[v], dd[b])))
        M = np.max(np.divide(pb, qb, out=np.zeros_like(pb), where=pb > 0))
        for _ in range(10000):
            v = r.choice(len(qb), p=qb)
            if r.random() * M * qb[v] <= pb[v]:
                break
        a_rej.append(float(np.dot(xb[v], dd[b])))
    assert ks_2samp(a_exact, a_rej).pvalue > 1e-3
