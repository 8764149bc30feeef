"""Sampling spheres for the direction getters.

The reference tracks on DIPY's ``repulsion724`` sphere (``run_gpu_streamlines.py:317-320``):
724 vertices and 2,166 edges (``3V - 6``) of its convex-hull triangulation.
DIPY is not available here, so this module builds a sphere of the same kind from
the published method: electrostatic repulsion of ``V/2`` charges, each paired with
its antipode (Jones et al. 1999), mirrored to ``V`` vertices, then triangulated by
the convex hull.  The vertex count, edge count and antipodal symmetry match the
reference sphere; the exact coordinates are this project's own.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

_DATA_DIR = os.path.join(os.path.dirname(__file__), "data")


@dataclass
class Sphere:
    vertices: np.ndarray  # [V, 3] float64 unit vectors
    edges: np.ndarray     # [E, 2] int32 vertex indices
    faces: np.ndarray     # [F, 3] int32

    @property
    def theta(self):
        return np.arccos(np.clip(self.vertices[:, 2], -1.0, 1.0))

    @property
    def phi(self):
        return np.arctan2(self.vertices[:, 1], self.vertices[:, 0])

    @property
    def x(self):
        return self.vertices[:, 0]

    @property
    def y(self):
        return self.vertices[:, 1]

    @property
    def z(self):
        return self.vertices[:, 2]


def _repulsion_hemisphere(n: int, iters: int = 2000, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    step = 0.05
    for it in range(iters):
        force = np.zeros_like(p)
        for sgn in (1.0, -1.0):
            d = p[:, None, :] - sgn * p[None, :, :]
            r2 = (d * d).sum(-1)
            if sgn > 0:
                np.fill_diagonal(r2, np.inf)
            inv3 = r2 ** -1.5
            force += (d * inv3[..., None]).sum(1)
        # project the force onto the tangent plane and take a normalised step
        force -= (force * p).sum(1, keepdims=True) * p
        fn = np.linalg.norm(force, axis=1, keepdims=True).max()
        p = p + step * force / fn
        p /= np.linalg.norm(p, axis=1, keepdims=True)
        step *= 0.998
    # canonical hemisphere representative: z > 0 (ties broken by y, x)
    flip = (p[:, 2] < 0) | ((p[:, 2] == 0) & (p[:, 1] < 0))
    p[flip] *= -1
    return p


def _hull(vertices: np.ndarray):
    from scipy.spatial import ConvexHull

    hull = ConvexHull(vertices)
    faces = np.sort(hull.simplices, axis=1).astype(np.int32)
    e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [0, 2]]])
    e = np.unique(e, axis=0).astype(np.int32)
    return faces, e


def make_repulsion_sphere(nvert: int = 724, iters: int = 2000, seed: int = 0) -> Sphere:
    if nvert % 2:
        raise ValueError("nvert must be even (antipodally symmetric sphere)")
    hemi = _repulsion_hemisphere(nvert // 2, iters=iters, seed=seed)
    verts = np.concatenate([hemi, -hemi], axis=0)
    faces, edges = _hull(verts)
    if len(edges) != 3 * nvert - 6:
        raise RuntimeError(f"triangulation has {len(edges)} edges, expected {3 * nvert - 6}")
    return Sphere(verts, edges, faces)


def get_sphere(name: str = "repulsion724") -> Sphere:
    """Return a cached repulsion sphere (``repulsion724`` or ``repulsion100``)."""
    sizes = {"repulsion724": 724, "repulsion200": 200, "repulsion100": 100}
    if name not in sizes:
        raise ValueError(f"unknown sphere {name!r}; choose one of {sorted(sizes)}")
    n = sizes[name]
    path = os.path.join(_DATA_DIR, f"{name}.npz")
    if os.path.exists(path):
        z = np.load(path)
        return Sphere(z["vertices"], z["edges"], z["faces"])
    s = make_repulsion_sphere(n)
    os.makedirs(_DATA_DIR, exist_ok=True)
    np.savez(path, vertices=s.vertices, edges=s.edges, faces=s.faces)
    return s
