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
