"""FA map and seeds on the GPU (csl_dti_fa, csl_seeds_from_mask) against the
float64 WLS restatement and the seeding distribution.

Bars: FA within 1e-6 of float64 (both fit in double from the same float32
signals); masked voxels 0.  Seeds: every seed's nearest voxel lies in the
mask, jitter in [-0.5, 0.5), voxels hit uniformly (chi-square p > 1e-4),
identical for the same generator seed, different for another.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dti_fa_matches_float64_wls():
    from gpustreamlines_b200.prep import dti_fa_gpu
    from oracle import cases, fp64

    ph = cases.phantom("csa_s")
    gt = ph.gtab
    mask = (ph.fa > 0.05).astype(np.float32)
    ref = fp64.dti_fa_wls(ph.dwi, gt.bvals, gt.bvecs, mask=mask)
    got = dti_fa_gpu(ph.dwi, gt.bvals, gt.bvecs, mask=mask).numpy()
    assert np.abs(got - ref).max() <= 1e-6
    assert (got[mask == 0] == 0).all()
    assert got.max() > 0.5


def test_seeds_from_mask_distribution():
    from scipy.stats import chisquare

    from gpustreamlines_b200.prep import seeds_from_mask_gpu
    from oracle import cases

    fa = cases.phantom("prob_s").fa
    n = 200000
    s = seeds_from_mask_gpu(fa, n, threshold=0.3, seed=7).numpy()
    v = np.floor(s + 0.5).astype(np.int64)
    assert (fa[v[:, 0], v[:, 1], v[:, 2]] > 0.3).all()
    frac = s - v
    assert (frac >= -0.5).all() and (frac < 0.5).all()
    vox = np.argwhere(fa > 0.3)
    lin = np.ravel_multi_index(v.T, fa.shape)
    counts = np.bincount(np.searchsorted(np.ravel_multi_index(vox.T, fa.shape), lin), minlength=len(vox))
    assert chisquare(counts).pvalue > 1e-4
    s2 = seeds_from_mask_gpu(fa, n, threshold=0.3, seed=7).numpy()
    s3 = seeds_from_mask_gpu(fa, n, threshold=0.3, seed=8).numpy()
    assert np.array_equal(s, s2) and not np.array_equal(s, s3)
    with pytest.raises(ValueError):
        seeds_from_mask_gpu(fa, 10, threshold=2.0)
