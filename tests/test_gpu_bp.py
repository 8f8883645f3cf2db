"""Backprojection on the GPU through the C ABI, against the oracle and the reference kernel.

FP32_EXACT must be bit-identical to the reference kernel cudaFdkBP (emulated by the oracle,
and the reference's own kernel compiled for sm_100a).  FP32 (staged) must match the
reference arithmetic within rel-L2 1e-5; MIXED (FP16 views) within rel-L2 1e-3 of FP64."""
import os

import numpy as np
import pytest

import fdk_b200 as F
from oracle import oracle as O
from tests.helpers import (knife_edge_mask, max_rel, oracle_bp_f64, oracle_bp_ref32, oracle_filtered,
                           phantom_views, rel_l2, small_param)

pytestmark = pytest.mark.gpu

REF_BP = os.path.join(O.REF_DIR, "libref_gpu_bp.so")


def run_bp(precision, p, top, bot, batches, mats_batches, transpose=1, width=None, height=None):
    width = width or p.nv
    height = height or p.nu
    bp = F.BackProjectionFDK(width, height, 32, p.nx, p.ny, p.nz, F.BoxT(*top), F.BoxT(*bot), precision)
    for f, m in zip(batches, mats_batches):
        bp.BP(transpose, f, width, height, m, f.shape[0])
    vol = bp.GetVolumeData()
    n, ms = bp.stats()
    assert n == sum(f.shape[0] for f in batches) and ms > 0
    bp.close()
    return vol


def random_views(n, h, w, seed=0):
    return np.random.default_rng(seed).standard_normal((n, h, w)).astype(np.float32)


@pytest.mark.parametrize("n,nu,nv,views", [(32, 40, 36, 16), (48, 64, 64, 40), (30, 33, 31, 7)])
def test_exact_symmetric_bitwise_vs_oracle(n, nu, nv, views):
    p = small_param(n, nu, nv, views)
    mats = p.proj_matrices()
    filt = random_views(views, nu, nv, seed=n)
    top = [0, 0, 0, n, n, n // 2]
    bot = [0, 0, n - n // 2, n, n, n // 2]
    batches = [filt[i:i + 32] for i in range(0, views, 32)]
    mb = [mats[i:i + 32] for i in range(0, views, 32)]
    got = run_bp("fp32_exact", p, top, bot, batches, mb)
    want = oracle_bp_ref32(top, bot[5], n, batches, mb)
    assert np.array_equal(got, want), (np.abs(got - want).max(), np.abs(want).max())


def test_exact_subbox_and_nonsymmetric_bitwise():
    n, views = 40, 12
    p = small_param(n, 48, 44, views)
    mats = p.proj_matrices()
    filt = random_views(views, 48, 44, seed=5)
    top = [4, 6, 8, 20, 24, 10]
    bot = [4, 6, n - 1 - 8 - 10 + 1, 20, 24, 10]
    got = run_bp("fp32_exact", p, top, bot, [filt], [mats])
    assert np.array_equal(got, oracle_bp_ref32(top, bot[5], n, [filt], [mats]))
    top2 = [0, 0, 5, n, n, 17]
    got2 = run_bp("fp32_exact", p, top2, [0, 0, 0, 0, 0, 0], [filt], [mats])
    assert np.array_equal(got2, oracle_bp_ref32(top2, 0, n, [filt], [mats]))


def test_exact_untransposed_views_bitwise():
    n, views = 32, 9
    p = small_param(n, 40, 36, views)
    mats = p.proj_matrices()
    filt_t = random_views(views, 40, 36, seed=9)           # (nu rows, nv)
    filt_r = np.ascontiguousarray(filt_t.transpose(0, 2, 1))  # (nv rows, nu)
    top = [0, 0, 0, n, n, n // 2]
    bot = [0, 0, n // 2, n, n, n // 2]
    a = run_bp("fp32_exact", p, top, bot, [filt_t], [mats], 1)
    b = run_bp("fp32_exact", p, top, bot, [filt_r], [mats], 0, width=40, height=36)
    # TRANSPOSE=0 blends along u first (the frame row), TRANSPOSE=1 along v first: same
    # samples, different rounding order
    assert rel_l2(b, a) <= 1e-6


@pytest.mark.skipif(not os.path.exists(REF_BP), reason="reference GPU build absent")
@pytest.mark.parametrize("views", [32, 45])
def test_exact_bitwise_vs_reference_kernel(views):
    """Against the reference's own cudaFdkBP compiled for sm_100a (BackProjectionFDK)."""
    n = 64
    p = small_param(n, 48, 40, views)
    mats = p.proj_matrices()
    filt = random_views(views, 48, 40, seed=11)
    top = [0, 0, 0, n, n, n // 2]
    bot = [0, 0, n // 2, n, n, n // 2]
    batches = [filt[i:i + 32] for i in range(0, views, 32)]
    mb = [mats[i:i + 32] for i in range(0, views, 32)]
    ref = O.RefGPU().backproject(batches, mb, n, n, n, top, bot)
    got = run_bp("fp32_exact", p, top, bot, batches, mb)
    assert np.array_equal(got, ref)
    assert np.array_equal(ref, oracle_bp_ref32(top, bot[5], n, batches, mb))  # pins the oracle


@pytest.mark.parametrize("kernel", ["tma", "staged"])
@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("mixed", 1e-3)])
@pytest.mark.parametrize("n,views", [(32, 24), (64, 64), (96, 40)])
def test_fast_paths_on_phantom(precision, tol, n, views, kernel, monkeypatch):
    """Both staged kernels: the TMA-fed persistent kernel and the synchronous-staging one."""
    if kernel == "staged":
        monkeypatch.setenv("FDK_BP_KERNEL", "staged")
    p = small_param(n, n, n, views)
    mats = p.proj_matrices()
    _, proj = phantom_views(p, seed=n)
    filt = oracle_filtered(p, proj)
    top = [0, 0, 0, n, n, n // 2]
    bot = [0, 0, n // 2, n, n, n // 2]
    batches = [filt[i:i + 32] for i in range(0, views, 32)]
    mb = [mats[i:i + 32] for i in range(0, views, 32)]
    got = run_bp(precision, p, top, bot, batches, mb)
    ref32 = oracle_bp_ref32(top, bot[5], n, batches, mb)
    f64, _ = oracle_bp_f64(top, bot[5], n, filt, p.proj_matrices(np.float64))
    m = knife_edge_mask(p, top, bot[5])
    e32, e64 = rel_l2(got[m], ref32[m]), rel_l2(got[m], f64[m])
    print(f"{precision} n={n}: rel-L2 vs reference arithmetic {e32:.2e}, vs FP64 {e64:.2e}, "
          f"max rel {max_rel(got, f64):.2e}")
    if precision == "fp32":
        assert e32 <= tol
    assert e64 <= tol


@pytest.mark.parametrize("kernel", ["tma", "staged"])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("nu,nv", [(24, 20), (26, 21)])  # nv=21: rows not 16-byte multiples
def test_fast_border_views(precision, kernel, nu, nv, monkeypatch):
    """Detector smaller than the volume's shadow: boundary samples follow SUBPIXEL's rule."""
    if kernel == "staged":
        monkeypatch.setenv("FDK_BP_KERNEL", "staged")
    n, views = 32, 16
    p = small_param(n, nu, nv, views)  # detector crops the volume in u and v
    p.du = p.dv = 384.0 / 40
    mats = p.proj_matrices()
    filt = random_views(views, nu, nv, seed=21)
    top = [0, 0, 0, n, n, n // 2]
    bot = [0, 0, n // 2, n, n, n // 2]
    got = run_bp(precision, p, top, bot, [filt], [mats])
    want = oracle_bp_ref32(top, bot[5], n, [filt], [mats])
    m = knife_edge_mask(p, top, bot[5])
    e = rel_l2(got[m], want[m])
    print(precision, kernel, nu, nv, "rel-L2 vs reference arithmetic", e)
    # MIXED on white-noise views: FP16 samples and the 1/1024-pixel fixed-point fraction of the
    # staged gather bound the per-sample error at a few 1e-4 of the sample differences; the
    # north-star bar of 1e-3 holds even here, where neighbouring samples are uncorrelated
    assert e <= (1e-5 if precision == "fp32" else 1e-3), e


def test_fast_rejects_non_circular_matrices():
    n = 16
    p = small_param(n, 16, 16, 4)
    mats = p.proj_matrices().copy()
    mats[:, 2] = 0.01
    bp = F.BackProjectionFDK(16, 16, 32, n, n, n, F.BoxT(0, 0, 0, n, n, 8), F.BoxT(0, 0, 8, n, n, 8), "fp32")
    with pytest.raises(F.FdkError):
        bp.BP(1, random_views(4, 16, 16), 16, 16, mats, 4)
