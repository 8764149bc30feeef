"""Float64 restatement of the bootstrap fit and the peak selection -- TEST
INFRASTRUCTURE ONLY (the accuracy reference for the FP32 and BF16x3 fits).

Follows the reference's sequence (boot.cu:393-608, tracking_helpers.cu:4-245,
boot.cu:115-193) in double precision from the same float32 inputs:
trilinear interpolation of the DWI (tracking_helpers.cu:4-61; outside the
half-voxel border the ODF is zero), hat/residual products over the non-b0
volumes, bootstrap h[j] + r[idx[j]], clamp at min_signal, division by the
mean clamped b0 signal, the CSA transform log(-log(clip(x, .001, .999))) with
coefficient 0 fixed at 1/(2 sqrt(pi)) or the OPDT form, the sphere sampling,
then the 5 % threshold, local maxima over the edges, the relative threshold,
the descending sort, the minimum-separation filter and the closest peak.
"""

from __future__ import annotations

import math

import numpy as np

N0 = 0.5 / math.sqrt(math.pi)


def trilinear(data: np.ndarray, pts: np.ndarray):
    """[n, T] float64 values and an in-bounds mask (same border rule as the kernels)."""
    X, Y, Z, T = data.shape
    p = np.asarray(pts, dtype=np.float64)
    inb = np.all(np.isfinite(p), axis=1)
    for a, dim in enumerate((X, Y, Z)):
        inb &= (p[:, a] >= -0.5) & (p[:, a] + 0.5 < dim)
    out = np.zeros((len(p), T))
    fl = np.floor(p)
    w1 = p - fl
    lo = np.clip(fl, 0, None).astype(np.int64)
    hi = np.minimum(lo + 1, np.array([X - 1, Y - 1, Z - 1]))
    idx = np.nonzero(inb)[0]
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                cx = (lo if i == 0 else hi)[idx, 0]
                cy = (lo if j == 0 else hi)[idx, 1]
                cz = (lo if k == 0 else hi)[idx, 2]
                w = ((1 - w1[idx, 0]) if i == 0 else w1[idx, 0]) * \
                    ((1 - w1[idx, 1]) if j == 0 else w1[idx, 1]) * \
                    ((1 - w1[idx, 2]) if k == 0 else w1[idx, 2])
                out[idx] += w[:, None] * data[cx, cy, cz].astype(np.float64)
    return out, inb


def boot_odf(inp: dict, model: str, pts: np.ndarray, resample: np.ndarray) -> np.ndarray:
    """[n, V] float64 ODFs of one bootstrap fit per point with the given resample indices."""
    b0 = np.asarray(inp["b0s_mask"]).astype(bool)
    nb = ~b0
    H = np.asarray(inp["H"], np.float64)
    R = np.asarray(inp["R"], np.float64)
    dq = np.asarray(inp["delta_q"], np.float64)
    db = np.asarray(inp["delta_b"], np.float64)
    S = np.asarray(inp["sampling_matrix"], np.float64)
    ms = float(inp.get("min_signal", 1.0))
    vals, inb = trilinear(inp["dataf"], pts)
    s = vals[:, nb]
    r = s @ R.T
    h = s @ H.T
    boot = h + np.take_along_axis(r, np.asarray(resample, np.int64), axis=1)
    full = vals.copy()
    full[:, nb] = boot
    full = np.maximum(ms, full)
    denom = full[:, b0].mean(axis=1)
    full = full / denom[:, None]
    y = full[:, nb]
    if model == "CSA":
        t = np.log(-np.log(np.clip(y, 0.001, 0.999)))
        coef = t @ dq.T
        coef[:, 0] = N0
    else:
        t1 = -np.log(y) * (1.5 + np.log(y)) * y
        coef = t1 @ dq.T - y @ db.T
    odf = coef @ S.T
    odf[~inb] = 0.0
    return odf


def peaks(odf: np.ndarray, verts: np.ndarray, edges: np.ndarray, rel: float, cos_min_sep: float,
          pmf_thr: float = 0.05, sphere_symm: bool = False) -> list[int]:
    """Kept peak vertices of one ODF row, in the reference's order."""
    o = np.asarray(odf, np.float64).copy()
    m = o.max()
    o[o < pmf_thr * m] = 0.0
    odf_min = max(0.0, o.min())
    a, b = edges[:, 0], edges[:, 1]
    flag = np.zeros(len(o), np.int64)
    less_a = o[a] < o[b]
    less_b = o[b] < o[a]
    gt = np.zeros(len(o), bool)
    lt = np.zeros(len(o), bool)
    np.logical_or.at(gt, a[less_a], True)
    np.logical_or.at(lt, b[less_a], True)
    np.logical_or.at(gt, b[less_b], True)
    np.logical_or.at(lt, a[less_b], True)
    flag[lt] = 1
    flag[gt] = -1
    mx = np.nonzero(flag > 0)[0]
    if len(mx) == 0:
        return []
    mm = (o[mx] - odf_min).max()
    keep = [v for v in mx if (o[v] - odf_min) >= rel * mm]
    if len(keep) < 32:
        keep = sorted(keep, key=lambda v: (-o[v], v))
    kept = [keep[0]] if keep else []
    for v in keep[1:]:
        ok = True
        for k in kept:
            cs = float(np.dot(verts[v], verts[k]))
            if sphere_symm:
                cs = abs(cs)
            if cs > cos_min_sep:
                ok = False
                break
        if ok:
            kept.append(v)
    return kept


def closest_peak(kept: list[int], verts: np.ndarray, direction: np.ndarray, cos_max: float):
    """(vertex, sign) of the peak the reference steps to, or None."""
    best, bdot = -1, 0.0
    for v in kept:
        d = float(np.dot(direction, verts[v]))
        if abs(d) > abs(bdot):
            best, bdot = v, d
    if best < 0:
        return None
    if bdot >= cos_max:
        return best, 1
    if bdot <= -cos_max:
        return best, -1
    return None


def dti_fa_wls(dwi, bvals, bvecs, mask=None, min_signal=1e-6):
    """FA from the weighted least-squares tensor fit (dipy.reconst.dti WLS:
    OLS on log signals, weights w = exp(X beta_ols), then the least-squares fit
    of w X beta = w y), eigenvalues clipped at 0, in float64."""
    b = np.asarray(bvals, np.float64)
    g = np.asarray(bvecs, np.float64)
    X = np.stack([np.ones_like(b), -b * g[:, 0] ** 2, -b * g[:, 1] ** 2, -b * g[:, 2] ** 2,
                  -2 * b * g[:, 0] * g[:, 1], -2 * b * g[:, 0] * g[:, 2], -2 * b * g[:, 1] * g[:, 2]], 1)
    P = np.linalg.inv(X.T @ X) @ X.T
    shp = dwi.shape[:3]
    y = np.log(np.maximum(np.asarray(dwi, np.float64).reshape(-1, dwi.shape[-1]), min_signal))
    b0 = y @ P.T
    w2 = np.exp(b0 @ X.T) ** 2
    A = np.einsum("nt,ti,tj->nij", w2, X, X)
    r = np.einsum("nt,ti,nt->ni", w2, X, y)
    beta = np.linalg.solve(A, r[..., None])[..., 0]
    D = np.empty((len(beta), 3, 3))
    D[:, 0, 0], D[:, 1, 1], D[:, 2, 2] = beta[:, 1], beta[:, 2], beta[:, 3]
    D[:, 0, 1] = D[:, 1, 0] = beta[:, 4]
    D[:, 0, 2] = D[:, 2, 0] = beta[:, 5]
    D[:, 1, 2] = D[:, 2, 1] = beta[:, 6]
    ev = np.clip(np.linalg.eigvalsh(D), 0, None)
    md = ev.mean(1, keepdims=True)
    num = np.sqrt(((ev - md) ** 2).sum(1))
    den = np.sqrt((ev ** 2).sum(1))
    fa = np.clip(np.sqrt(1.5) * np.where(den > 0, num / np.where(den > 0, den, 1), 0), 0, 1)
    if mask is not None:
        fa = np.where(np.asarray(mask).reshape(-1) > 0, fa, 0)
    return fa.reshape(shp)
