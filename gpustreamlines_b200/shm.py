"""Float64 spherical-harmonic model matrices for the bootstrap direction getter.

The reference builds these through DIPY (``cuslines/boot_utils.py:8-94``):
``shm.real_sh_descoteaux(legacy=True)``, ``OpdtModel._fit_matrix``,
``CsaOdfModel._fit_matrix``, ``shm.hat`` and ``shm.lcr_matrix``.  DIPY is a
third-party dependency that is not vendored with the reference (its version
is unpinned in ``pyproject.toml``), so this module restates the published
mathematics directly:

* real, even-order SH basis of Descoteaux et al. 2007 ("legacy" sign
  convention: ``m > 0`` uses the imaginary part, ``m < 0`` the real part of
  ``Y_l^|m|``, both scaled by sqrt(2));
* CSA fit matrix of Aganj et al. 2010: ``(P_l(0) * -l(l+1)) / (8 pi) * pinv``;
* OPDT fit matrices of Tristan-Vega et al. 2009:
  ``delta_b = P_l(0) * -l(l+1) * pinv`` and ``delta_q = 4 P_l(0) * pinv``;
* Laplace-Beltrami regularised pseudo-inverse ``pinv([B; sqrt(lambda) L])``;
* hat matrix ``H = U U^T`` of the thin SVD of ``B`` and leveraged, centred
  residual matrix ``R = D (I - H) - mean_rows(D (I - H))`` with
  ``D = diag(1 / sqrt(1 - h_ii))`` (residual bootstrap, Berman et al. 2008).

All arithmetic is float64; the tracker casts the results to float32 exactly
as the reference does (``cu_direction_getters.py:168-175``).
"""

from __future__ import annotations

import numpy as np
from scipy import special


def sph_harm_ind_list(sh_order_max: int, full_basis: bool = False):
    """Return ``(m_values, l_values)`` in the order l ascending, m = -l..l."""
    if sh_order_max % 2 != 0 and not full_basis:
        raise ValueError("sh_order_max must be an even integer")
    step = 1 if full_basis else 2
    ls = np.arange(0, sh_order_max + 1, step)
    m_list, l_list = [], []
    for l in ls:
        for m in range(-l, l + 1):
            m_list.append(m)
            l_list.append(l)
    return np.asarray(m_list, dtype=int), np.asarray(l_list, dtype=int)


def cart2sphere(x, y, z):
    """Cartesian to (r, theta=polar, phi=azimuth)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64)
    r = np.sqrt(x * x + y * y + z * z)
    with np.errstate(invalid="ignore", divide="ignore"):
        theta = np.arccos(np.where(r > 0, z / np.where(r > 0, r, 1.0), 1.0))
    theta = np.where(r > 0, theta, 0.0)
    phi = np.arctan2(y, x)
    return r, theta, phi


def _complex_sh(m_abs, l, theta, phi):
    """Complex orthonormal Y_l^m (Condon-Shortley phase) at polar theta, azimuth phi."""
    return special.sph_harm_y(l, m_abs, theta, phi)


def real_sh_descoteaux(sh_order_max, theta, phi, full_basis=False, legacy=True):
    """Real SH basis (Descoteaux 2007) sampled at (theta, phi).

    Returns ``(B, m_values, l_values)`` with ``B`` of shape ``[npoints, ncoef]``.
    """
    m_values, l_values = sph_harm_ind_list(sh_order_max, full_basis)
    theta = np.asarray(theta, dtype=np.float64).reshape(-1, 1)
    phi = np.asarray(phi, dtype=np.float64).reshape(-1, 1)
    if legacy:
        sh = _complex_sh(np.abs(m_values), l_values, theta, phi)
    else:
        # non-legacy: negative orders use Y_l^{-m} directly
        sh = _complex_sh(np.abs(m_values), l_values, theta, phi)
        sh = np.where(m_values < 0, np.conj(sh) * (-1.0) ** np.abs(m_values), sh)
    real = np.where(m_values > 0, sh.imag, sh.real)
    real = real * np.where(m_values == 0, 1.0, np.sqrt(2.0))
    return real, m_values, l_values


def smooth_pinv(B, L):
    """Regularised pseudo-inverse: ``pinv([B; diag(L)])[:, :len(B)]``."""
    Lm = np.diag(L)
    inv = np.linalg.pinv(np.concatenate((B, Lm)))
    return inv[:, : len(B)]


def hat(B):
    """Hat (projection) matrix of the least-squares fit with design ``B``."""
    U, _, _ = np.linalg.svd(B, full_matrices=False)
    return U @ U.T


def lcr_matrix(H):
    """Leveraged, centred residual matrix of the residual bootstrap."""
    H = np.asarray(H, dtype=np.float64)
    if H.ndim != 2 or H.shape[0] != H.shape[1]:
        raise ValueError("H should be a square matrix")
    d = H.diagonal()
    lev = np.ones_like(d)
    ok = d < 1
    lev[ok] = 1.0 / np.sqrt(1.0 - d[ok])
    R = (np.eye(len(H)) - H) * lev[:, None]
    return R - R.mean(0)


def _legendre_at_zero(l_values):
    return special.eval_legendre(l_values, 0.0)


class _GradientTable:
    """Minimal duck-typed gradient table (bvals, bvecs, b0s_mask, gradients)."""

    def __init__(self, bvals, bvecs, b0_threshold=50.0):
        self.bvals = np.asarray(bvals, dtype=np.float64)
        self.bvecs = np.asarray(bvecs, dtype=np.float64)
        self.b0_threshold = b0_threshold
        self.b0s_mask = self.bvals <= b0_threshold

    @property
    def gradients(self):
        return self.bvals[:, None] * self.bvecs


def gradient_table(bvals, bvecs, b0_threshold=50.0):
    return _GradientTable(bvals, bvecs, b0_threshold)


def _dwi_design(gtab, sh_order_max, full_basis=False):
    b0s = np.asarray(gtab.b0s_mask, dtype=bool)
    grads = getattr(gtab, "gradients", None)
    if grads is None:  # a duck-typed table with bvals / bvecs only (DIPY: gradients = bvals * bvecs)
        grads = np.asarray(gtab.bvals, dtype=np.float64)[:, None] * np.asarray(gtab.bvecs, dtype=np.float64)
    grads = np.asarray(grads, dtype=np.float64)[~b0s]
    _, theta, phi = cart2sphere(grads[:, 0], grads[:, 1], grads[:, 2])
    B, m_values, l_values = real_sh_descoteaux(sh_order_max, theta, phi, full_basis, legacy=True)
    return B, m_values, l_values


def csa_fit_matrix(gtab, sh_order_max=6, smooth=0.006):
    B, _, l_values = _dwi_design(gtab, sh_order_max)
    L = -l_values * (l_values + 1.0)
    F = _legendre_at_zero(l_values)
    invB = smooth_pinv(B, np.sqrt(smooth) * L)
    return (F * L)[:, None] / (8.0 * np.pi) * invB


def opdt_fit_matrices(gtab, sh_order_max=6, smooth=0.006):
    B, _, l_values = _dwi_design(gtab, sh_order_max)
    L = -l_values * (l_values + 1.0)
    F = _legendre_at_zero(l_values)
    invB = smooth_pinv(B, np.sqrt(smooth) * L)
    delta_b = (F * L)[:, None] * invB
    delta_q = 4.0 * F[:, None] * invB
    return delta_b, delta_q


def hat_and_lcr(gtab, sh_order_max):
    """H and R over the non-b0 directions (``boot_utils.py:86-94``)."""
    B, _, _ = _dwi_design(gtab, sh_order_max)
    H = hat(B)
    return H, lcr_matrix(H)


def _sphere_angles(sphere):
    if hasattr(sphere, "theta") and hasattr(sphere, "phi"):
        return np.asarray(sphere.theta), np.asarray(sphere.phi)
    v = np.asarray(sphere.vertices, dtype=np.float64)
    _, theta, phi = cart2sphere(v[:, 0], v[:, 1], v[:, 2])
    return theta, phi


def prepare_opdt(gtab, sphere, sh_order_max=6, full_basis=False, sh_lambda=0.006, min_signal=1):
    """Bootstrap matrices for the OPDT model (``boot_utils.py:11-45``)."""
    theta, phi = _sphere_angles(sphere)
    sampling_matrix, _, _ = real_sh_descoteaux(sh_order_max, theta, phi, full_basis, legacy=True)
    delta_b, delta_q = opdt_fit_matrices(gtab, sh_order_max, sh_lambda)
    H, R = hat_and_lcr(gtab, sh_order_max)
    return dict(model_type="OPDT", min_signal=min_signal, H=H, R=R,
                delta_b=delta_b, delta_q=delta_q,
                sampling_matrix=sampling_matrix, b0s_mask=np.asarray(gtab.b0s_mask))


def prepare_csa(gtab, sphere, sh_order_max=6, full_basis=False, sh_lambda=0.006, min_signal=1):
    """Bootstrap matrices for the CSA model (``boot_utils.py:48-83``)."""
    theta, phi = _sphere_angles(sphere)
    sampling_matrix, _, _ = real_sh_descoteaux(sh_order_max, theta, phi, full_basis, legacy=True)
    fit = csa_fit_matrix(gtab, sh_order_max, sh_lambda)
    H, R = hat_and_lcr(gtab, sh_order_max)
    return dict(model_type="CSA", min_signal=min_signal, H=H, R=R,
                delta_b=fit, delta_q=fit,
                sampling_matrix=sampling_matrix, b0s_mask=np.asarray(gtab.b0s_mask))
