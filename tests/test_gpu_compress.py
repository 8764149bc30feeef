"""Streamline linearisation on the device (csl_compress) against the host
restatement (io.compress_streamlines after Tractogram.to_world), on tracked
prob_s streamlines.

Bars: with an identity or a diagonal affine (exact in float32) the kept
points are bit-identical; with a general rotation + shear affine (float64
products whose last-bit rounding may differ between the device and BLAS) at
least 99.5 % of streamlines are identical and the rest differ only where a
point sits on the tolerance boundary; length filtering drops the same
streamlines.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_parity import _handle

pytestmark = pytest.mark.gpu


def _tracked(n=800):
    from oracle import cases

    seeds = cases.seeds("prob_s", n, seed=21)
    h = _handle("prob_s")
    h.propagate(seeds)
    L, S, P = h.fetch()
    return h, L, P


def _host(L, P, affine, tol, maxseg, minlen=0, maxlen=np.inf):
    from gpustreamlines_b200.io import ArraySequence, Tractogram, compress_streamlines

    keep = (L >= minlen) & (L <= maxlen)
    off = np.concatenate([[0], np.cumsum(L)])
    parts = [P[off[i]:off[i + 1]] for i in range(len(L)) if keep[i]]
    seq = ArraySequence(parts)
    t = Tractogram(seq, affine_to_rasmm=affine).to_world()
    return compress_streamlines(list(t.streamlines), tol_error=tol, max_segment_length=maxseg)


def _device(h, affine, tol, maxseg, minlen=0, maxlen=None):
    cnt, pts = h.compress(affine, tol, maxseg, minlen, maxlen)
    off = np.concatenate([[0], np.cumsum(cnt[cnt > 0])])
    return [pts[off[i]:off[i + 1]] for i in range(len(off) - 1)]


@pytest.mark.parametrize("affine", ["eye", "diag"])
def test_compress_bit_exact(affine):
    h, L, P = _tracked()
    try:
        A = np.eye(4) if affine == "eye" else np.diag([2.0, 2.0, 2.5, 1.0])
        for tol, maxseg in ((0.1, 10.0), (0.01, 3.0)):
            host = _host(L, P, A, tol, maxseg)
            dev = _device(h, A, tol, maxseg)
            assert len(host) == len(dev) == len(L)
            for a, b in zip(host, dev):
                assert a.shape == b.shape and np.array_equal(a.astype(np.float32), b)
            assert sum(len(x) for x in dev) < P.shape[0]
    finally:
        h.close()


def test_compress_general_affine_and_filter():
    h, L, P = _tracked()
    try:
        rng = np.random.default_rng(3)
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        A = np.eye(4)
        A[:3, :3] = Q @ np.diag([2.0, 2.0, 2.0]) + 0.05 * rng.normal(size=(3, 3))
        A[:3, 3] = [-90.0, -126.0, -72.0]
        host = _host(L, P, A, 0.1, 10.0)
        dev = _device(h, A, 0.1, 10.0)
        same = [a.shape == b.shape and np.allclose(a, b, rtol=0, atol=1e-4) for a, b in zip(host, dev)]
        assert len(host) == len(dev) and np.mean(same) >= 0.995
        host = _host(L, P, A, 0.1, 10.0, minlen=10, maxlen=200)
        dev = _device(h, A, 0.1, 10.0, minlen=10, maxlen=200)
        assert len(host) == len(dev) == int(((L >= 10) & (L <= 200)).sum())
    finally:
        h.close()
