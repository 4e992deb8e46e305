"""Seeded synthetic inputs for the transforms (no external datasets).

* ``ellipsoid_phantom`` -- a sum of K seeded ellipsoids: centres uniform in the
  ball of radius 0.6, semi-axes U[0.05, 0.3], uniformly random rotations,
  densities U[-0.5, 1.0]; zero outside the unit ball.  Sampled at the nodes
  x_i = -1 + 2 i / (n - 1) of the reference's volume grid (the grid that
  radon_grid/src/interp.c:32 and ray_grid/src/interp.c:32 assume), in the
  reference's file order v[ix][iy][iz] (radon_grid/src/init.c:120-124).
* ``layer_frames`` -- the axis orientations of the layer-by-layer ray scheme:
  frame 0 is the identity (the reference's z-slices, ray_grid/src/ray_grid.c),
  the others are seeded uniformly random rotations.

The support of every phantom lies within radius 0.9 (0.6 + 0.3), i.e. inside
the unit ball that the reference assumes (radon_grid/src/radon_grid.c:30-31).
"""
from __future__ import annotations

import numpy as np


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Haar-uniform rotation matrix (QR of a Gaussian matrix, signs fixed)."""
    a = rng.standard_normal((3, 3))
    q, r = np.linalg.qr(a)
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def ellipsoid_params(k: int, rng: np.random.Generator):
    """Centres, semi-axes, rotations and densities of k ellipsoids."""
    centres = np.empty((k, 3))
    for i in range(k):  # uniform in the ball of radius 0.6
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        centres[i] = d * 0.6 * rng.random() ** (1.0 / 3.0)
    axes = rng.uniform(0.05, 0.3, size=(k, 3))
    rots = np.stack([random_rotation(rng) for _ in range(k)])
    dens = rng.uniform(-0.5, 1.0, size=k)
    return centres, axes, rots, dens


def ellipsoid_phantom(n: int, k: int, seed: int, dtype=np.float64) -> np.ndarray:
    """n^3 node-sampled phantom in v[ix][iy][iz] order.  Each ellipsoid is
    evaluated on the nodes of its bounding cube only (it lies within its
    largest semi-axis of its centre); densities add in ellipsoid order."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres, axes, rots, dens = ellipsoid_params(k, rng)
    t = -1.0 + 2.0 * np.arange(n) / (n - 1)
    out = np.zeros((n, n, n), dtype=np.float64)
    for c, a, R, rho in zip(centres, axes, rots, dens):
        r = a.max()
        lo = np.searchsorted(t, c - r, side="left")
        hi = np.searchsorted(t, c + r, side="right")
        x = np.stack(np.meshgrid(t[lo[0]:hi[0]], t[lo[1]:hi[1]], t[lo[2]:hi[2]], indexing="ij"),
                     axis=-1)
        local = (x - c) @ R  # R^T (x - c) for each node
        q = np.sum((local / a) ** 2, axis=-1)
        out[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += np.where(q <= 1.0, rho, 0.0)
    r2 = t[:, None, None] ** 2 + t[None, :, None] ** 2 + t[None, None, :] ** 2
    out[r2 > 1.0] = 0.0
    return out.astype(dtype, copy=False)


def layer_frames(count: int, seed: int) -> np.ndarray:
    """(count, 3, 3) rotation frames; frame 0 is the identity."""
    rng = np.random.Generator(np.random.PCG64(seed))
    frames = [np.eye(3)]
    for _ in range(count - 1):
        frames.append(random_rotation(rng))
    return np.ascontiguousarray(np.stack(frames))
