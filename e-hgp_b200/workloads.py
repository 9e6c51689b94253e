"""Seeded synthetic point clouds with the shapes of the product path's workloads.

No public dataset is involved; every generator is PCG64-seeded and returns an
(n, 3) array (float64 or float32 as the workload states).  Duplicate points
are re-drawn, because the canonical point cloud rejects duplicates
(morsehgp3d/src/cpu/spatial/point_cloud.cpp:64-71).
"""
from __future__ import annotations

import numpy as np


def _dedupe(pts: np.ndarray, redraw, rng) -> np.ndarray:
    """Re-draws rows that duplicate an earlier row (bitwise on +0-canonical values)."""
    for _ in range(100):
        canon = pts + 0.0  # -0 -> +0
        view = np.ascontiguousarray(canon).view(np.dtype((np.void, canon.dtype.itemsize * 3))).ravel()
        _, first = np.unique(view, return_index=True)
        dup = np.ones(len(pts), bool)
        dup[first] = False
        if not dup.any():
            return pts
        pts[dup] = redraw(int(dup.sum()), rng)
    raise RuntimeError("could not remove duplicates")


def uniform_cube(n: int = 256, seed: int = 0) -> np.ndarray:
    """n i.i.d. U[0,1]^3 points, binary64 (the plain one-cloud workload, n=256)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    draw = lambda k, r: r.random((k, 3))
    return _dedupe(draw(n, rng), draw, rng)


def jittered_lattice(side: int = 37, seed: int = 0, jitter: float = 0.25) -> np.ndarray:
    """side^3 unit-lattice points, each axis jittered by U[-jitter, jitter], stored
    as binary32 (37^3 = 50,653 points is the regular volumetric workload)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = np.arange(side, dtype=np.float64)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pts = (lat + rng.uniform(-jitter, jitter, lat.shape)).astype(np.float32)
    redraw = lambda k, r: (r.uniform(0, side - 1, (k, 3))).astype(np.float32)
    return _dedupe(pts, redraw, rng)


def _haar_rotation(rng) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def clustered(n: int = 200_000, seed: int = 0, components: int = 8, background: float = 0.2,
              snapped: float = 0.05, dtype=np.float64) -> np.ndarray:
    """Anisotropic Gaussian mixture (means U[0,10]^3, covariance eigenvalues
    log-uniform in [0.05, 1], Haar rotations) plus a uniform background; a
    fraction of all points snapped to the 2^-10 grid to force exact ties."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_bg = int(round(background * n))
    n_cl = n - n_bg
    means = rng.uniform(0, 10, (components, 3))
    covs = []
    for _ in range(components):
        lam = np.exp(rng.uniform(np.log(0.05), np.log(1.0), 3))
        R = _haar_rotation(rng)
        covs.append(R @ np.diag(lam) @ R.T)
    labels = rng.integers(0, components, n_cl)
    pts = np.empty((n, 3))
    for c in range(components):
        idx = np.nonzero(labels == c)[0]
        pts[idx] = rng.multivariate_normal(means[c], covs[c], len(idx))
    pts[n_cl:] = rng.uniform(0, 10, (n_bg, 3))
    snap = rng.random(n) < snapped
    pts[snap] = np.round(pts[snap] * 1024.0) / 1024.0
    pts = pts.astype(dtype)
    redraw = lambda k, r: r.uniform(0, 10, (k, 3)).astype(dtype)
    return _dedupe(pts, redraw, rng)


def mixture_cloud(n: int, rng, dtype=np.float32) -> np.ndarray:
    """Gaussian mixture of 1-6 components plus 10% uniform noise (batched workload)."""
    k = int(rng.integers(1, 7))
    n_noise = int(round(0.1 * n))
    means = rng.uniform(0, 10, (k, 3))
    scales = np.exp(rng.uniform(np.log(0.2), np.log(1.5), k))
    lab = rng.integers(0, k, n - n_noise)
    pts = np.empty((n, 3))
    pts[: n - n_noise] = means[lab] + rng.standard_normal((n - n_noise, 3)) * scales[lab, None]
    pts[n - n_noise:] = rng.uniform(0, 10, (n_noise, 3))
    pts = pts.astype(dtype)
    redraw = lambda m, r: r.uniform(0, 10, (m, 3)).astype(dtype)
    return _dedupe(pts, redraw, rng)


def batched_uneven(count: int = 512, seed: int = 0, lo: int = 1000, hi: int = 20000) -> list[np.ndarray]:
    """`count` independent clouds, sizes log-uniform in [lo, hi], FP32."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    return [mixture_cloud(int(s), rng) for s in sizes]
