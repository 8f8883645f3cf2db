"""Pin the CPU oracle against the reference's own code compiled from its sources
(oracle/_ref/libref_cpu.so, built by oracle/build_ref.sh) and against known answers.

The reference ships no golden vectors or known-answer tests, so this is the pin."""
import os

import numpy as np
import pytest

from fdk_b200 import config
from oracle import oracle as O

REF_CPU = os.path.join(O.REF_DIR, "libref_cpu.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU build absent")


def small(n=32, views=16):
    p = config("c1")
    p.nx = p.ny = p.nz = n
    p.dx = p.dy = p.dz = 256.0 / n
    p.nu = p.nv = n
    p.du = p.dv = 384.0 / n
    p.nProj = views
    return p


@needs_ref
@pytest.mark.parametrize("ftype", ["none", "ram-lak", "shepp-logan", "cosine", "hamming", "hann"])
@pytest.mark.parametrize("nu", [60, 64, 256, 1536])
def test_filter_design_matches_reference(ftype, nu):
    p = small()
    p.nu = nu
    ref = O.RefCPU().parameter(p, ftype)["H"]
    assert np.array_equal(O.filter_design(ftype, nu), ref)


@needs_ref
@pytest.mark.parametrize("cfg", ["c1", "c4"])
def test_cos_table_matches_reference_bitwise(cfg):
    p = config(cfg)
    p.nProj = 8
    p.offset_nu, p.offset_nv = 1.25, -0.5
    ref = O.RefCPU().parameter(p)["cos"]
    assert np.array_equal(O.cos_table(p), ref)


@needs_ref
def test_proj_matrices_match_reference():
    p = small(views=24)
    p.volume_postion_angle = 0.3
    ref = O.RefCPU().parameter(p)["mats"].astype(np.float64)
    m = O.proj_matrices(p)
    # the reference forms the product in FP32; the oracle in FP64
    assert np.abs(m - ref).max() <= 4e-7 * np.abs(m).max()
    assert np.all(m[:, 2] == 0) and np.all(m[:, 10] == 0)  # circular orbit: no z term in rows 0, 2


@needs_ref
@pytest.mark.parametrize("shape", [(16, 64), (7, 60), (32, 256)])
def test_filter_rows_match_reference_bourke(shape):
    """Oracle row filter (pad = mean of 3) == the reference's double-precision filterImageRow."""
    rng = np.random.default_rng(1)
    src = rng.standard_normal(shape).astype(np.float32)
    H = O.filter_design("hann", shape[1])
    ref = O.RefCPU().filter_rows(H, src)
    got = O.filter_view(src, H, None, pad_n=3)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_fma_rz_known_answers():
    L = O.lib()
    f = np.float32
    assert L.orc_fma_rz(1.0, 1.0, 1e-8) == 1.0  # 1 + 1e-8 rounds toward zero to 1
    assert L.orc_fma_rz(-1.0, 1.0, -1e-8) == -1.0
    assert np.float32(L.orc_fma_rz(1.0, 1.0, -1e-8)) == np.nextafter(f(1.0), f(0.0))
    assert np.float32(L.orc_fma_rz(-1.0, 1.0, 1e-8)) == -np.nextafter(f(1.0), f(0.0))
    # exact results are unchanged
    assert L.orc_fma_rz(3.0, 5.0, 7.0) == 22.0
    rng = np.random.default_rng(0)
    for _ in range(2000):
        a, b, c = (rng.standard_normal(3) * 10 ** rng.uniform(-3, 3, 3)).astype(np.float32)
        r = np.float32(L.orc_fma_rz(float(a), float(b), float(c)))
        exact = float(a) * float(b) + float(c)  # a*b exact in double; sum rounds at 2^-53
        # r is the float toward zero of the exact value: |r| <= |exact| < |r| + ulp
        assert abs(float(r)) <= abs(exact) * (1 + 2 ** -50)
        nxt = np.nextafter(r, np.float32(np.inf) if exact > 0 else np.float32(-np.inf))
        assert abs(float(nxt)) >= abs(exact) * (1 - 2 ** -50)


@needs_ref
def test_3dct_cpu_fdk_matches_oracle_pipeline():
    """The reference's CPU FDK (3dct BackProjection) / AngularAndrampFactor equals the oracle's
    FP64 filter (pad 3) + FP64 backprojection, away from the detector border where the two
    bilinear boundary rules differ (type.h:2196-2207 vs backprojectionFDK.cu:18)."""
    n = 48
    p = small(n, views=24)
    ell = np.array([[12.0, -20.0, 10.0, 60.0, 40.0, 50.0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 1.0]])
    proj = np.stack([O.ellipsoid_projection(ell, p, a) for a in O.view_angles(p)])
    H = O.filter_design("hann", p.nu)
    cos = O.cos_table(p)
    filt = np.stack([O.filter_view(v, H, cos, pad_n=3, transpose=True) for v in proj])
    vol = np.zeros(n * n * n)
    O.bp_f64(vol, [0, 0, 0, n, n, n // 2], n // 2, n, filt, O.proj_matrices(p))
    rec = O.transform_volume(vol.astype(np.float32), n, n, n)
    ref = np.zeros((n, n, n), np.float32)
    O.RefCPU().cpu_fdk(p, proj, 0, ref)
    ref /= O.angular_ramp_factor(p)
    zz, yy, xx = np.meshgrid(*(np.arange(n) - (n - 1) / 2,) * 3, indexing="ij")
    core = (xx ** 2 + yy ** 2 < (0.35 * n) ** 2) & (np.abs(zz) < 0.35 * n)
    err = np.linalg.norm((rec - ref)[core]) / np.linalg.norm(ref[core])
    assert err < 2e-4, err


@needs_ref
@pytest.mark.parametrize("n,nu,nv,views", [(48, 56, 40, 6), (64, 64, 64, 9)])
def test_forward_projector_matches_reference(n, nu, nv, views):
    """The oracle's ray marcher (orc_forward_project, the learned filter's training-data
    projector) against the reference's own 3dct ForwardProjection<float> (3dct/3dct.cpp:430-573,
    angle as CTForwardProjection forms it, :594), built from its sources: same rays, box, step and
    trilinear samples, FP32 in a different order."""
    from fdk_b200.phantom import phantom_for
    from tests.helpers import small_param

    p = small_param(n, nu, nv, views)
    vol = O.ellipsoid_volume(phantom_for(p, 4, 12), p)
    R = O.RefCPU()
    for i, a in enumerate(O.view_angles(p)):
        ref = R.forward_projection(vol, p, i)
        got = O.forward_project(vol, p, a)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 2e-5, i
        assert np.abs(got - ref).max() <= 5e-5 * np.abs(ref).max(), i
