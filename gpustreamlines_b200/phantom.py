"""Seeded synthetic diffusion phantom that stands in for the Stanford HARDI data.

The reference benchmarks on Stanford HARDI (81x106x76 voxels, 10 b0 + 150
directions at b=2000; ``cuslines/webgpu/README.md:31``).  That dataset is not
available offline, so this module generates a phantom with the same shapes and
value ranges:

* curved tube bundles (arcs, a commissural sweep and a sinusoid) that cross at
  roughly 60-90 degrees inside an ellipsoidal brain mask;
* a two-fibre cylindrically-symmetric multi-tensor signal with eigenvalues
  (1.7e-3, 0.3e-3, 0.3e-3) mm^2/s, an isotropic 0.8e-3 mm^2/s background,
  S0 = 100 and Rician noise at SNR 20;
* FA from this module's own log-linear least-squares tensor fit;
* an ODF/PMF volume on a sphere built from the true fibre directions with a
  sharpened order-8 SH kernel plus small SH noise, clipped at zero (the
  reference's CSD ODF is clipped the same way, ``run_gpu_streamlines.py:378``);
* seeds drawn uniformly from the FA > 0.3 mask with a uniform voxel jitter.

Everything is driven by one numpy PCG64 seed, so the same call reproduces the
same arrays bit for bit.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import shm
from .sphere import get_sphere

LAMBDA_PAR = 1.7e-3
LAMBDA_PERP = 0.3e-3
D_ISO = 0.8e-3


@dataclass
class Phantom:
    shape: tuple
    voxel_mm: float
    bvals: np.ndarray
    bvecs: np.ndarray
    dwi: np.ndarray | None          # [X,Y,Z,T] float32
    fa: np.ndarray                  # [X,Y,Z] float32
    mask: np.ndarray                # [X,Y,Z] bool brain mask
    fiber_dirs: np.ndarray          # [X,Y,Z,2,3] float32 (zero where absent)
    fiber_frac: np.ndarray          # [X,Y,Z,2] float32
    sh_coef: np.ndarray | None = None   # [X,Y,Z,C] float32 ODF SH coefficients
    meta: dict = field(default_factory=dict)

    @property
    def gtab(self):
        return shm.gradient_table(self.bvals, self.bvecs)


def _hemisphere_dirs(n, rng):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[v[:, 2] < 0] *= -1
    return v


def _bundle_curves(shape):
    """Centre lines (in voxel coordinates) of the synthetic bundles."""
    X, Y, Z = shape
    t = np.linspace(0.0, 1.0, 400)
    curves = []
    # 1) arc in the x-y plane (corpus-callosum-like commissural sweep across x = X/2)
    ang = np.pi * (0.15 + 0.7 * t)
    curves.append(np.stack([X / 2 + 0.38 * X * np.cos(ang),
                            0.30 * Y + 0.35 * Y * np.sin(ang),
                            0.55 * Z + 0.08 * Z * np.sin(2 * np.pi * t)], 1))
    # 2) front-back bundle along y with a gentle bend in z (crosses the arc)
    curves.append(np.stack([0.35 * X + 0.04 * X * np.sin(np.pi * t),
                            0.05 * Y + 0.9 * Y * t,
                            0.35 * Z + 0.25 * Z * np.sin(np.pi * t)], 1))
    # 3) mirrored front-back bundle on the other hemisphere
    curves.append(np.stack([0.65 * X - 0.04 * X * np.sin(np.pi * t),
                            0.05 * Y + 0.9 * Y * t,
                            0.35 * Z + 0.25 * Z * np.sin(np.pi * t)], 1))
    # 4) inferior-superior bundle, tilted, crossing bundles 2 and the arc
    curves.append(np.stack([0.30 * X + 0.40 * X * t,
                            0.55 * Y + 0.10 * Y * np.sin(2 * np.pi * t),
                            0.08 * Z + 0.84 * Z * t], 1))
    # 5) sinusoid along x at low z
    curves.append(np.stack([0.08 * X + 0.84 * X * t,
                            0.62 * Y + 0.12 * Y * np.sin(2 * np.pi * t),
                            0.30 * Z + 0.05 * Z * np.cos(2 * np.pi * t)], 1))
    return curves


def _rasterize_bundles(shape, radius):
    """Per voxel, the two closest bundle tangents within ``radius`` voxels."""
    X, Y, Z = shape
    n = X * Y * Z
    best_d = np.full((n, 2), np.inf)
    best_dir = np.zeros((n, 2, 3))
    for c in _bundle_curves(shape):
        tang = np.gradient(c, axis=0)
        tang /= np.linalg.norm(tang, axis=1, keepdims=True)
        dist = np.full(n, np.inf)
        tdir = np.zeros((n, 3))
        r = int(np.ceil(radius)) + 1
        for p, tv in zip(c, tang):
            lo = np.maximum(np.floor(p - r).astype(int), 0)
            hi = np.minimum(np.ceil(p + r).astype(int) + 1, [X, Y, Z])
            if np.any(hi <= lo):
                continue
            gx, gy, gz = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]),
                                     np.arange(lo[2], hi[2]), indexing="ij")
            d = np.sqrt((gx - p[0]) ** 2 + (gy - p[1]) ** 2 + (gz - p[2]) ** 2).ravel()
            idx = ((gx * Y + gy) * Z + gz).ravel()
            upd = d < dist[idx]
            dist[idx[upd]] = d[upd]
            tdir[idx[upd]] = tv
        inside = dist < radius
        # insert into the 2-slot nearest list
        for slot in (0, 1):
            better = inside & (dist < best_d[:, slot])
            if slot == 0:
                best_d[better, 1] = best_d[better, 0]
                best_dir[better, 1] = best_dir[better, 0]
            best_d[better, slot] = dist[better]
            best_dir[better, slot] = tdir[better]
            inside = inside & ~better
    return best_d.reshape(X, Y, Z, 2), best_dir.reshape(X, Y, Z, 2, 3)


def _tensor_fa(dwi, bvals, bvecs, mask):
    """Log-linear least-squares DTI fit -> FA (float32)."""
    g = bvecs
    b = bvals
    A = np.stack([np.ones_like(b), -b * g[:, 0] ** 2, -b * g[:, 1] ** 2, -b * g[:, 2] ** 2,
                  -2 * b * g[:, 0] * g[:, 1], -2 * b * g[:, 0] * g[:, 2],
                  -2 * b * g[:, 1] * g[:, 2]], 1)
    P = np.linalg.pinv(A)  # [7, T]
    shp = dwi.shape[:3]
    flat = dwi.reshape(-1, dwi.shape[-1])
    m = mask.ravel()
    fa = np.zeros(flat.shape[0], dtype=np.float64)
    idx = np.nonzero(m)[0]
    for s in range(0, len(idx), 65536):
        ii = idx[s:s + 65536]
        y = np.log(np.maximum(flat[ii].astype(np.float64), 1e-3))
        coef = y @ P.T
        D = np.empty((len(ii), 3, 3))
        D[:, 0, 0], D[:, 1, 1], D[:, 2, 2] = coef[:, 1], coef[:, 2], coef[:, 3]
        D[:, 0, 1] = D[:, 1, 0] = coef[:, 4]
        D[:, 0, 2] = D[:, 2, 0] = coef[:, 5]
        D[:, 1, 2] = D[:, 2, 1] = coef[:, 6]
        ev = np.clip(np.linalg.eigvalsh(D), 0, None)
        md = ev.mean(1, keepdims=True)
        num = np.sqrt(((ev - md) ** 2).sum(1))
        den = np.sqrt((ev ** 2).sum(1))
        fa[ii] = np.sqrt(1.5) * np.where(den > 0, num / np.where(den > 0, den, 1), 0)
    return np.clip(fa, 0, 1).reshape(shp).astype(np.float32)


def make_phantom(shape=(81, 106, 76), seed=1234, n_b0=10, n_dirs=150, bval=2000.0,
                 snr=20.0, s0=100.0, voxel_mm=2.0, with_dwi=True, sh_order=8,
                 odf_sharpness=0.05, odf_noise=0.02) -> Phantom:
    """Build the phantom (see module docstring).  ``seed`` feeds numpy's PCG64."""
    rng = np.random.default_rng(seed)
    X, Y, Z = shape
    bvecs = np.concatenate([np.zeros((n_b0, 3)), _hemisphere_dirs(n_dirs, rng)])
    bvals = np.concatenate([np.zeros(n_b0), np.full(n_dirs, bval)])

    gx, gy, gz = np.meshgrid(np.arange(X), np.arange(Y), np.arange(Z), indexing="ij")
    ell = (((gx - (X - 1) / 2) / (0.48 * X)) ** 2 + ((gy - (Y - 1) / 2) / (0.48 * Y)) ** 2
           + ((gz - (Z - 1) / 2) / (0.48 * Z)) ** 2)
    mask = ell <= 1.0

    radius = max(2.5, 0.07 * min(shape))
    dist, fdirs = _rasterize_bundles(shape, radius)
    present = np.isfinite(dist) & mask[..., None]
    frac = np.where(present, 1.0, 0.0)
    nf = frac.sum(-1, keepdims=True)
    fib_total = np.where(nf > 0, 0.85, 0.0)
    frac = np.where(nf > 0, frac / np.maximum(nf, 1) * fib_total, 0.0)
    f_iso = np.where(mask, 1.0 - frac.sum(-1), 0.0)
    fdirs = np.where(present[..., None], fdirs, 0.0)

    dwi = None
    if with_dwi:
        T = len(bvals)
        dwi = np.zeros((X * Y * Z, T), dtype=np.float32)
        fl_frac = frac.reshape(-1, 2)
        fl_dirs = fdirs.reshape(-1, 2, 3)
        fl_iso = f_iso.ravel()
        sigma = s0 / snr
        for s in range(0, X * Y * Z, 65536):
            sl = slice(s, s + 65536)
            sig = fl_iso[sl, None] * np.exp(-bvals * D_ISO)[None, :]
            for k in range(2):
                cos2 = (fl_dirs[sl, k, :] @ bvecs.T) ** 2
                adc = LAMBDA_PERP + (LAMBDA_PAR - LAMBDA_PERP) * cos2
                sig = sig + fl_frac[sl, k, None] * np.exp(-bvals[None, :] * adc)
            sig *= s0
            n1 = rng.normal(0, sigma, sig.shape)
            n2 = rng.normal(0, sigma, sig.shape)
            dwi[sl] = np.sqrt((sig + n1) ** 2 + n2 ** 2).astype(np.float32)
        dwi = dwi.reshape(X, Y, Z, T)
        fa = _tensor_fa(dwi, bvals, bvecs, mask)
    else:
        # analytic FA of the noiseless mixture (used only when no DWI is requested)
        fa = _analytic_fa(frac, fdirs, f_iso)
        fa = np.where(mask, fa, 0).astype(np.float32)

    # ODF SH coefficients: sharpened delta kernel per fibre + isotropic part + noise
    m_vals, l_vals = shm.sph_harm_ind_list(sh_order)
    kern = np.exp(-odf_sharpness * l_vals * (l_vals + 1.0))
    ncoef = len(l_vals)
    coef = np.zeros((X * Y * Z, ncoef), dtype=np.float64)
    fl_frac = frac.reshape(-1, 2)
    fl_dirs = fdirs.reshape(-1, 2, 3)
    for k in range(2):
        has = fl_frac[:, k] > 0
        if not np.any(has):
            continue
        _, th, ph = shm.cart2sphere(fl_dirs[has, k, 0], fl_dirs[has, k, 1], fl_dirs[has, k, 2])
        Bd, _, _ = shm.real_sh_descoteaux(sh_order, th, ph)
        coef[has] += fl_frac[has, k, None] * Bd * kern[None, :]
    coef[:, 0] += f_iso.ravel() * 0.5 / np.sqrt(np.pi) * 0.3
    inb = mask.ravel()
    coef[inb] += rng.normal(0, odf_noise, (int(inb.sum()), ncoef)) * (l_vals > 0)
    coef[~inb] = 0
    coef = coef.reshape(X, Y, Z, ncoef).astype(np.float32)

    return Phantom(shape=shape, voxel_mm=voxel_mm, bvals=bvals, bvecs=bvecs, dwi=dwi,
                   fa=fa, mask=mask, fiber_dirs=fdirs.astype(np.float32),
                   fiber_frac=frac.astype(np.float32), sh_coef=coef,
                   meta=dict(seed=seed, rng="numpy.PCG64", snr=snr, s0=s0, bval=bval,
                             sh_order=sh_order))


def _analytic_fa(frac, fdirs, f_iso):
    D = f_iso[..., None, None] * D_ISO * np.eye(3)
    for k in range(2):
        d = fdirs[..., k, :]
        D = D + frac[..., k, None, None] * (LAMBDA_PERP * np.eye(3)
                                            + (LAMBDA_PAR - LAMBDA_PERP) * d[..., :, None] * d[..., None, :])
    tot = (f_iso + frac.sum(-1))[..., None, None]
    D = np.where(tot > 0, D / np.where(tot > 0, tot, 1), 0)
    ev = np.linalg.eigvalsh(D.reshape(-1, 3, 3))
    md = ev.mean(1, keepdims=True)
    num = np.sqrt(((ev - md) ** 2).sum(1))
    den = np.sqrt((ev ** 2).sum(1))
    fa = np.sqrt(1.5) * np.where(den > 0, num / np.where(den > 0, den, 1), 0)
    return fa.reshape(frac.shape[:3])


def odf_volume(ph: Phantom, sphere=None, out=None, chunk=65536) -> np.ndarray:
    """Evaluate the phantom ODF on ``sphere`` -> float32 [X,Y,Z,V], clipped >= 0."""
    sphere = sphere or get_sphere("repulsion724")
    B, _, _ = shm.real_sh_descoteaux(ph.meta["sh_order"], sphere.theta, sphere.phi)
    Bt = B.T.astype(np.float32)
    coef = ph.sh_coef.reshape(-1, ph.sh_coef.shape[-1])
    n = coef.shape[0]
    V = Bt.shape[1]
    if out is None:
        out = np.empty((n, V), dtype=np.float32)
    else:
        out = out.reshape(n, V)
    for s in range(0, n, chunk):
        np.matmul(coef[s:s + chunk], Bt, out=out[s:s + chunk])
        np.maximum(out[s:s + chunk], 0, out=out[s:s + chunk])
    return out.reshape(*ph.shape, V)


def seeds_from_mask(fa, n, threshold=0.3, seed=0):
    """Seeds uniform over voxels with ``fa > threshold`` plus U[-0.5, 0.5)^3 jitter."""
    rng = np.random.default_rng(seed)
    vox = np.argwhere(fa > threshold)
    if len(vox) == 0:
        raise ValueError("empty seed mask")
    pick = vox[rng.integers(0, len(vox), n)]
    return (pick + rng.uniform(-0.5, 0.5, (n, 3))).astype(np.float64)
