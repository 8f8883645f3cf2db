"""Shared test fixtures: small geometries, phantom-based filtered views, error metrics."""
import numpy as np

import fdk_b200 as F
from oracle import oracle as O


def small_param(n=32, nu=None, nv=None, views=16, cfg="c1"):
    """c1's geometry (SOD 1000, SID 1500, 256 mm FOV, 384 mm detector) at n^3 / nu x nv."""
    p = F.config(cfg)
    nu = nu or n
    nv = nv or n
    p.nx = p.ny = p.nz = n
    p.dx = p.dy = p.dz = 256.0 / n
    p.nu, p.nv = nu, nv
    p.du = 384.0 / nu
    p.dv = 384.0 / nu
    p.nProj = views
    return p


def phantom_views(p, seed=3, n_ell=12):
    """Exact projections (oracle, FP64) of a seeded random-ellipsoid phantom: (views, nv, nu)."""
    from fdk_b200.phantom import phantom_for

    ell = phantom_for(p, seed, n_ell)
    return ell, np.stack([O.ellipsoid_projection(ell, p, a) for a in O.view_angles(p)])


def oracle_filtered(p, proj, pad_n=4):
    """Oracle FP64 filter (cosine weight, pad, Hann ramp), transposed: (views, nu, nv) f32."""
    H = O.filter_design(p.str_filter, p.nu)
    cos = O.cos_table(p)
    return np.stack([O.filter_view(v, H, cos, pad_n=pad_n, transpose=True) for v in proj])


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def oracle_bp_ref32(top, depth_bottom, nz, filt_batches, mats_batches):
    """Oracle volume after the reference kernel's sequence of launches: [zs][y][x]."""
    D = top[5] + depth_bottom
    vol = np.zeros(top[3] * top[4] * D, np.float32)
    for f, m in zip(filt_batches, mats_batches):
        O.bp_ref32(vol, top, depth_bottom, nz, f, m)
    return O.transform_volume(vol, top[3], top[4], D)


def oracle_bp_f64(top, depth_bottom, nz, filt, mats64):
    D = top[5] + depth_bottom
    vol = np.zeros(top[3] * top[4] * D, np.float64)
    O.bp_f64(vol, top, depth_bottom, nz, filt, mats64)
    return O.transform_volume(vol.astype(np.float32), top[3], top[4], D), vol


def knife_edge_mask(p, top, depth_bottom, eps=1e-3):
    """Voxels (in [zs][y][x] storage order of the slab pair) whose projection in some view
    lands within eps pixels of a detector border (u or v at 0 or n-1).  The reference's
    bilinear rule (backprojectionFDK.cu:18) zeroes a sample at u, v >= n-1 and keeps it just
    below, so at the border any change of FP32 rounding switches a whole sample on or off.
    Parity between different FP32 arithmetics is measured on the other voxels."""
    mats = p.proj_matrices(np.float64)
    D = top[5] + depth_bottom
    zs = np.concatenate([np.arange(top[2], top[2] + top[5]),
                         np.arange(p.nz - top[2] - depth_bottom, p.nz - top[2])]) if depth_bottom else \
        np.arange(top[2], top[2] + top[5])
    z, y, x = np.meshgrid(zs.astype(np.float64), np.arange(top[1], top[1] + top[4], dtype=np.float64),
                          np.arange(top[0], top[0] + top[3], dtype=np.float64), indexing="ij")
    bad = np.zeros(z.shape, bool)
    for m in mats:
        w = m[8] * x + m[9] * y + m[10] * z + m[11]
        u = (m[0] * x + m[1] * y + m[2] * z + m[3]) / w
        v = (m[4] * x + m[5] * y + m[6] * z + m[7]) / w
        for c, n in ((u, p.nu), (v, p.nv)):
            bad |= (np.abs(c) < eps) | (np.abs(c - (n - 1)) < eps)
    return ~bad
