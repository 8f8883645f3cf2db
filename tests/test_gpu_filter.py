"""Ramp filter on the GPU against the FP64 oracle and the reference's cuFFT plugin."""
import os

import numpy as np
import pytest

import fdk_b200 as F
from oracle import oracle as O
from tests.helpers import max_rel, phantom_views, small_param

pytestmark = pytest.mark.gpu
REF_FLT = os.path.join(O.REF_DIR, "libref_gpu_filter.so")


@pytest.mark.parametrize("nu,nv", [(64, 64), (256, 256), (96, 50), (1536, 16), (2048, 8)])
@pytest.mark.parametrize("transpose", [False, True])
def test_filter_engine_vs_oracle(nu, nv, transpose):
    p = small_param(64, nu, nv, 4)
    rng = np.random.default_rng(nu + nv)
    src = (rng.standard_normal((nv, nu)) * 50 + 100).astype(np.float32)
    cos = p.cos_sigma
    eng = F.FilterEngine(cos, p.fft_kernel_real_f32)
    want = O.filter_view(src, p.fft_kernel_real, cos, pad_n=4, transpose=transpose)
    s = src.copy()
    dst = np.zeros((nu, nv) if transpose else (nv, nu), np.float32)
    eng.Filtering(s, dst, transpose)
    assert np.array_equal(s, src * cos)  # src is cosine-weighted in place, in FP32
    assert max_rel(dst, want) <= 2e-6, max_rel(dst, want)


@pytest.mark.parametrize("nu,nv", [(80, 64), (96, 50), (2048, 16), (300, 24)])
def test_device_layouts(nu, nv):
    """All device layouts against the FP64 oracle and each other.  nv = 64 and 16 take the grouped
    MIRROR kernel (row pairs tiled 2 or 4 at a time), nv = 50 the per-pair fallback, nv = 24 the
    grouped FP32 and fallback FP16 kernels."""
    import torch

    p = small_param(64, nu, nv, 6)
    _, proj = phantom_views(p)
    eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32)
    src = torch.from_numpy(proj).cuda()
    want = np.stack([O.filter_view(v, p.fft_kernel_real, p.cos_sigma, pad_n=4, transpose=True) for v in proj])
    t = torch.empty((6, nu, nv), dtype=torch.float32, device="cuda")
    eng.run_device(src.data_ptr(), t.data_ptr(), 6, F.LAYOUT_TRANSPOSED, F.DTYPE_F32)
    m = torch.empty((6, nu, nv, 2), dtype=torch.float32, device="cuda")
    eng.run_device(src.data_ptr(), m.data_ptr(), 6, F.LAYOUT_MIRROR, F.DTYPE_F32)
    h = torch.empty((6, nu, nv, 2), dtype=torch.float16, device="cuda")
    scale = float(1.0 / p.cos_sigma.max())  # back to line-integral units, inside the FP16 range
    eng.run_device(src.data_ptr(), h.data_ptr(), 6, F.LAYOUT_MIRROR, F.DTYPE_F16, scale)
    r = torch.empty((6, nv, nu), dtype=torch.float32, device="cuda")
    eng.run_device(src.data_ptr(), r.data_ptr(), 6, F.LAYOUT_ROWS, F.DTYPE_F32)
    torch.cuda.synchronize()
    t, m, h, r = t.cpu().numpy(), m.cpu().numpy(), h.float().cpu().numpy() / scale, r.cpu().numpy()
    # FP32 FFT rounding grows with log2(W): 12 radix-2 stages each way at W = 4096
    assert max_rel(t, want) <= (2e-6 if nu <= 1024 else 3e-6)
    assert np.array_equal(r.transpose(0, 2, 1), t)
    assert np.array_equal(m[..., 0], t) and np.array_equal(m[..., 1], t[:, :, ::-1])
    assert max_rel(h[..., 0], want) <= 1e-3 and max_rel(h[..., 1], want[:, :, ::-1]) <= 1e-3


@pytest.mark.skipif(not os.path.exists(REF_FLT), reason="reference GPU build absent")
@pytest.mark.parametrize("nu,nv", [(64, 64), (512, 32), (256, 100)])
def test_cufft_plugin_api_vs_reference(nu, nv):
    """correct_image_real32 + filter_row_real32 == the reference's CorrectImage_Real32 +
    FilterRow_Real32 (cuFFT, pad 3) on the same device buffers."""
    import torch

    p = small_param(64, nu, nv, 3)
    rng = np.random.default_rng(7)
    views = torch.from_numpy((rng.standard_normal((3, nv, nu)) * 10).astype(np.float32)).cuda()
    table = torch.from_numpy(p.cos_sigma).cuda()
    H = torch.from_numpy(p.fft_kernel_real_f32).cuda()
    ref = O.RefGPU().filter(views.clone(), table, H, len(H)).cpu().numpy()
    a = views.clone()
    F.correct_image_real32(a, table, a)
    out = torch.empty_like(a)
    F.filter_row_real32(a, out, H)
    got = out.cpu().numpy()
    want = np.stack([O.filter_view(v, p.fft_kernel_real, p.cos_sigma, pad_n=3) for v in views.cpu().numpy()])
    assert max_rel(ref, want) <= 5e-6  # reference vs oracle
    assert max_rel(got, ref) <= 5e-6, max_rel(got, ref)


@pytest.mark.parametrize("nu,nv", [(512, 512), (1024, 64)])
def test_mirror_kernel_at_the_48k_shared_memory_boundary(nu, nv):
    """nu = 512 (W = 1024, four pairs at once) and nu = 1024 (W = 2048, two pairs) put the grouped
    MIRROR kernel at exactly 48 KiB of dynamic shared memory for FP16 and FP32 outputs."""
    import torch

    p = small_param(64, nu, nv, 2)
    rng = np.random.default_rng(nu)
    src = torch.from_numpy((rng.standard_normal((2, nv, nu)) * 10 + 40).astype(np.float32)).cuda()
    eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32)
    t = torch.empty((2, nu, nv), dtype=torch.float32, device="cuda")
    eng.run_device(src.data_ptr(), t.data_ptr(), 2, F.LAYOUT_TRANSPOSED, F.DTYPE_F32)
    m = torch.empty((2, nu, nv, 2), dtype=torch.float32, device="cuda")
    eng.run_device(src.data_ptr(), m.data_ptr(), 2, F.LAYOUT_MIRROR, F.DTYPE_F32)
    h = torch.empty((2, nu, nv, 2), dtype=torch.float16, device="cuda")
    scale = float(1.0 / p.cos_sigma.max())
    eng.run_device(src.data_ptr(), h.data_ptr(), 2, F.LAYOUT_MIRROR, F.DTYPE_F16, scale)
    torch.cuda.synchronize()
    t, m = t.cpu().numpy(), m.cpu().numpy()
    assert np.array_equal(m[..., 0], t) and np.array_equal(m[..., 1], t[:, :, ::-1])
    hh = h.float().cpu().numpy() / scale
    assert max_rel(hh[..., 0], t) <= 1e-3
