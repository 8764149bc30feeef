"""Streamline statistics for comparing trackings (host numpy).

``streamline_stats`` restates the reference benchmark's metric collection
(``cuslines/webgpu/benchmark.py:209-235``: count, mean / median / min / max
points per streamline, and commissural streamlines -- those whose x
coordinate crosses the volume's midline ``dimx / 2`` in voxel space).  The
voxel-density comparisons are the usual tractogram-overlap measures: binary
Dice of the visited-voxel sets and the overlap of the normalised visit
densities (1 - total-variation distance).
"""

from __future__ import annotations

import numpy as np


def _split_x(lengths: np.ndarray, points: np.ndarray):
    off = np.concatenate([[0], np.cumsum(lengths, dtype=np.int64)])
    return off


def streamline_stats(lengths, points, dimx: int) -> dict:
    """Reference statistics of one tractogram in voxel coordinates."""
    lengths = np.asarray(lengths, dtype=np.int64)
    n = len(lengths)
    if n == 0:
        return {"n_streamlines": 0}
    pts = np.asarray(points, dtype=np.float32).reshape(-1, 3)
    off = _split_x(lengths, pts)
    midx = dimx / 2.0
    x = pts[:, 0]
    # per-streamline min / max of x, vectorised with reduceat (every length >= 1)
    xmin = np.minimum.reduceat(x, off[:-1])
    xmax = np.maximum.reduceat(x, off[:-1])
    comm = int(np.count_nonzero((xmin < midx) & (xmax > midx)))
    return {
        "n_streamlines": int(n),
        "mean_pts": float(lengths.mean()),
        "median_pts": float(np.median(lengths)),
        "min_pts": int(lengths.min()),
        "max_pts": int(lengths.max()),
        "commissural": comm,
    }


def voxel_density(points, shape) -> np.ndarray:
    """Points per voxel (nearest voxel centre), flattened [X*Y*Z] int64."""
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    X, Y, Z = shape
    v = np.floor(pts + 0.5).astype(np.int64)
    ok = (v[:, 0] >= 0) & (v[:, 0] < X) & (v[:, 1] >= 0) & (v[:, 1] < Y) & (v[:, 2] >= 0) & (v[:, 2] < Z)
    v = v[ok]
    flat = (v[:, 0] * Y + v[:, 1]) * Z + v[:, 2]
    return np.bincount(flat, minlength=X * Y * Z)


def dice(a: np.ndarray, b: np.ndarray) -> float:
    """Binary Dice coefficient of the voxels visited by two tractograms."""
    A, B = a > 0, b > 0
    s = int(A.sum() + B.sum())
    return 1.0 if s == 0 else 2.0 * int((A & B).sum()) / s


def density_overlap(a: np.ndarray, b: np.ndarray) -> float:
    """Overlap of the normalised visit densities: sum_v min(a_v / |a|, b_v / |b|)."""
    sa, sb = float(a.sum()), float(b.sum())
    if sa == 0 or sb == 0:
        return 1.0 if sa == sb else 0.0
    return float(np.minimum(a / sa, b / sb).sum())


def ks_2samp(x, y) -> tuple[float, float]:
    """Two-sample Kolmogorov-Smirnov statistic and asymptotic p-value."""
    from scipy import stats

    r = stats.ks_2samp(np.asarray(x), np.asarray(y))
    return float(r.statistic), float(r.pvalue)
