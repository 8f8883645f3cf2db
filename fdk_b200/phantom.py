"""Seeded random-ellipsoid phantoms and their exact projections (synthetic benchmark data).

Ellipsoid record (16 float64): centre (cx, cy, cz) mm, semi-axes (a, b, c) mm, rotation R
(row major, world = R @ local), density rho.  World frame = the projection matrices' frame:
X = (x-(nx-1)/2) dx, Y = -(y-(ny-1)/2) dy, Z = -(z-(nz-1)/2) dz.

Distribution (the benchmark's phantom spec): centres uniform in the ball of radius 0.8 R,
semi-axes uniform in [0.05, 0.4] R, uniformly random rotations (Z-Y-Z Euler angles with
cos(beta) uniform), densities uniform in [-0.2, 1.0], additive; R = half the volume side.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _rot_zyz(a: float, b: float, g: float) -> np.ndarray:
    def rz(t):
        c, s = np.cos(t), np.sin(t)
        return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])

    def ry(t):
        c, s = np.cos(t), np.sin(t)
        return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])

    return rz(a) @ ry(b) @ rz(g)


def random_ellipsoids(seed: int, n: int, radius_mm: float) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 16), np.float64)
    for k in range(n):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        r = 0.8 * radius_mm * rng.uniform() ** (1.0 / 3.0)
        centre = d * r
        axes = rng.uniform(0.05, 0.4, size=3) * radius_mm
        R = _rot_zyz(rng.uniform(0, 2 * np.pi), np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi))
        rho = rng.uniform(-0.2, 1.0)
        out[k, 0:3] = centre
        out[k, 3:6] = axes
        out[k, 6:15] = R.reshape(-1)
        out[k, 15] = rho
    return out


def phantom_for(param, seed: int, n: int) -> np.ndarray:
    return random_ellipsoids(seed, n, 0.5 * param.nx * param.dx)


def project(param, ell: np.ndarray, first: int, n: int, dev_out: int, stream: int = 0) -> None:
    """Exact line integrals of views [first, first+n) into device memory (nv x nu each, f32)."""
    e = np.ascontiguousarray(ell, np.float64)
    g = param.to_c()
    check(lib().fdk_phantom_project(C.byref(g), e.ctypes.data, len(e), first, n, dev_out, stream))


def voxelize(param, ell: np.ndarray) -> np.ndarray:
    """Ground-truth volume [z][y][x] (value at voxel centres), numpy, for small checks."""
    nz, ny, nx = param.nz, param.ny, param.nx
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    P = np.stack([(x - (nx - 1) / 2.0) * param.dx, -(y - (ny - 1) / 2.0) * param.dy,
                  -(z - (nz - 1) / 2.0) * param.dz], -1)
    vol = np.zeros((nz, ny, nx), np.float32)
    for e in ell:
        R = e[6:15].reshape(3, 3)
        loc = (P - e[0:3]) @ R  # R^T (p - c) as row vectors
        q = ((loc / e[3:6]) ** 2).sum(-1)
        vol += np.where(q <= 1.0, e[15], 0.0).astype(np.float32)
    return vol
