"""Scan presets and seeded synthetic phantoms shared by the tests and the bench.

The workloads stand in for the reference's measured datasets (absent: the
reference ships no projections, .gitignore:4-5): cone-beam geometry with
SOD 500 mm / SDD 1000 mm and 2 mm detector pixels, so the reference's derived
voxel size sod*det/sdd (geometry.h:13) is 1 mm.
"""
from __future__ import annotations

import numpy as np


def three_axes() -> np.ndarray:
    """Three sample-rotation axes: identity, then the two 90-degree tilts that
    put the rotation axis along x and along y (elemR, params.cu:31)."""
    return np.array([[1, 0, 0, 0, 1, 0, 0, 0, 1],
                     [0, 0, -1, 0, 1, 0, 1, 0, 0],
                     [1, 0, 0, 0, 0, -1, 0, 1, 0]], np.float32)


def basis13() -> np.ndarray:
    """13 unit scattering directions, one per antipodal pair of the cubic
    symmetry directions: 3 axes, 6 face diagonals, 4 body diagonals."""
    d = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1),
         (0, 1, 1), (0, 1, -1), (1, 1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1)]
    return np.array([np.asarray(v, np.float64) / np.linalg.norm(v) for v in d], np.float32)


def oblique_rot(seed: int, n: int) -> np.ndarray:
    """n rotation matrices in general position (not grid-aligned), rows of 9."""
    rng = np.random.default_rng(seed)
    return np.array([_rot_from(rng).ravel() for _ in range(n)], np.float32)


def _rot_from(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def ellipsoid_phantom(N: int, n_ell: int, seed: int) -> np.ndarray:
    """Additive random ellipsoids: centres and semi-axes uniform within 0.8 of
    the half field of view, random orientation, attenuation U[0.1, 1.0]."""
    rng = np.random.default_rng(seed)
    c = (np.arange(N) - (N - 1) / 2.0)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    P = np.stack([x, y, z], -1).reshape(-1, 3)
    vol = np.zeros(N ** 3, np.float32)
    half = 0.8 * N / 2.0
    for _ in range(n_ell):
        ctr = rng.uniform(-half, half, 3) * 0.5
        ax = rng.uniform(0.1, 1.0, 3) * half * 0.5
        R = _rot_from(rng)
        val = rng.uniform(0.1, 1.0)
        q = (P - ctr) @ R
        inside = ((q / ax) ** 2).sum(-1) <= 1.0
        vol[inside] += val
    return vol.reshape(N, N, N)


def fiber_phantom(N: int, n_fib: int, seed: int, basis: np.ndarray) -> np.ndarray:
    """Straight fiber cylinders (radius U[2,5] voxels, unit direction f uniform
    on the sphere, through a random point); channel k holds |S_k x f|^2 inside
    a fiber and 0 outside.  Returns (K, N, N, N) float32, z-slowest."""
    rng = np.random.default_rng(seed)
    K = basis.shape[0]
    c = (np.arange(N) - (N - 1) / 2.0)
    vol = np.zeros((K, N, N, N), np.float32)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    for _ in range(n_fib):
        f = rng.normal(size=3)
        f /= np.linalg.norm(f)
        p0 = rng.uniform(-0.3 * N, 0.3 * N, 3)
        r = rng.uniform(2.0, 5.0)
        dx, dy, dz = x - p0[0], y - p0[1], z - p0[2]
        t = dx * f[0] + dy * f[1] + dz * f[2]
        d2 = dx * dx + dy * dy + dz * dz - t * t
        inside = d2 <= r * r
        eta = np.sum(np.cross(basis.astype(np.float64), f[None, :]) ** 2, axis=1)
        for k in range(K):
            vol[k][inside] = eta[k]
    return vol
