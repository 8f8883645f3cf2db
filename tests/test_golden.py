"""The oracle, and the product's host geometry, against committed outputs of the reference's own
CPU code (tests/golden/ref_cpu.npz, written by tests/golden/make_golden.py from the reference
compiled from its sources).  These need neither the reference tree nor its build: the same
checks as tests/test_oracle_pin.py, pinned to fixed vectors."""
import os
import sys

import numpy as np
import pytest

import fdk_b200 as F
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as MG  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "ref_cpu.npz"))


@pytest.mark.parametrize("nu", [60, 64, 256])
@pytest.mark.parametrize("window", MG.WINDOWS)
def test_filter_response_equals_reference(window, nu):
    """filter() (common/type.h:4427-4475) with its window quirks: bit for bit, oracle and product."""
    want = G[f"H_{window}_{nu}"]
    assert np.array_equal(O.filter_design(window, nu), want)
    p = F.config("c1")
    p.nu = nu
    p.str_filter = window
    assert np.array_equal(p.fft_kernel_real, want)


def test_filter_response_at_w4096_equals_reference():
    assert np.array_equal(O.filter_design("hann", 1536), G["H_hann_1536"])


def test_cos_table_and_matrices_equal_reference():
    g = MG.cos_geometry()
    assert np.array_equal(O.cos_table(g), G["cos"])  # the oracle restates the FP32 table bit for bit
    p = F.config("c1")
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "du", "dv", "nProj", "offset_nu", "offset_nv",
              "volume_postion_angle"):
        setattr(p, k, getattr(g, k))
    assert np.abs(p.cos_sigma.view(np.int32) - G["cos"].view(np.int32)).max() <= 1  # product: FP64, one FP32 rounding
    ref = G["mats"].astype(np.float64)
    for m in (O.proj_matrices(g), p.proj_matrices(np.float64)):
        # the reference multiplies its six 4x4 matrices in FP32; oracle and product in FP64
        assert np.abs(m - ref).max() <= 4e-7 * np.abs(m).max()


def test_bourke_row_filter_equals_reference():
    got = O.filter_view(MG.rows_input(), G["rows_H"], None, pad_n=3)
    want = G["rows_out"]
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


def test_3dct_cpu_fdk_equals_oracle_pipeline():
    """3dct's CPU FDK / AngularAndrampFactor against the oracle's FP64 filter (pad 3) and FP64
    backprojection, inside the detector-covered core (the two bilinear boundary rules differ at
    the border: type.h:2196-2207 against backprojectionFDK.cu:18)."""
    p = MG.small(32, views=16)
    n = p.nx
    proj = MG.fdk_projections(p)
    assert np.abs(proj - G["fdk_proj"]).max() <= 1e-6 * np.abs(G["fdk_proj"]).max()  # inputs reproduced
    H = O.filter_design("hann", p.nu)
    cos = O.cos_table(p)
    filt = np.stack([O.filter_view(v, H, cos, pad_n=3, transpose=True) for v in G["fdk_proj"]])
    vol = np.zeros(n * n * n)
    O.bp_f64(vol, [0, 0, 0, n, n, n // 2], n // 2, n, filt, O.proj_matrices(p))
    rec = O.transform_volume(vol.astype(np.float32), n, n, n)
    ref = G["fdk_vol"] / O.angular_ramp_factor(p)
    zz, yy, xx = np.meshgrid(*(np.arange(n) - (n - 1) / 2,) * 3, indexing="ij")
    core = (xx ** 2 + yy ** 2 < (0.35 * n) ** 2) & (np.abs(zz) < 0.35 * n)
    err = np.linalg.norm((rec - ref)[core]) / np.linalg.norm(ref[core])
    assert err < 2e-4, err


def test_ray_marcher_equals_reference():
    """The oracle's ray marcher against 3dct ForwardProjection<float> (3dct/3dct.cpp:430-573)."""
    q = MG.fproj_geometry()
    v = MG.fproj_volume(q)
    for i, a in enumerate(O.view_angles(q)):
        want = G["fproj"][i]
        got = O.forward_project(v, q, a)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 2e-5, i
        assert np.abs(got - want).max() <= 5e-5 * np.abs(want).max(), i


import make_golden_gpu as MGG  # noqa: E402

GG = np.load(os.path.join(HERE, "golden", "ref_gpu.npz"))


def test_reference_cufft_filter_equals_oracle():
    """The cuFFT plugin (CorrectImage_Real32 + FilterRow_Real32, pad = mean of 3) as it ran on a
    B200, against the oracle's FP64 row filter with the same table and response."""
    views = MGG.filter_views()
    want = GG["flt_out"]
    H = GG["flt_H"].astype(np.float64)
    got = np.stack([O.filter_view(v, H, GG["flt_cos"], pad_n=3) for v in views])
    assert np.abs(got - want).max() <= 5e-6 * np.abs(want).max()
