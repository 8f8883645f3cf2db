"""fdk_filter_row_real32_noalloc: the row filter for callers that cannot allocate device memory
when they filter (they reserve the device budget up front, or must keep cudaMalloc/cudaFree,
which may synchronise the device, out of their processing loop).

The test calls the new entry point through the C ABI twice in a row (different sizes, so the
second call must rebuild the shared tables), each time against the existing allocating entry
point fdk_filter_row_real32 on the same inputs, within the filter tests' tolerance.  One more
case checks the tables it builds on the GPU (twiddles from sincospi, the bit-reversed response)
against the FP64 oracle's row filter (pad 3, the cuFFT plugin's edge rule).  It lives in a file
of its own that pytest collects last, and passes alone or after the other tests."""
import ctypes as C

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200._lib import DataRef, lib

pytestmark = pytest.mark.gpu

TOL = 5e-6  # max relative error, as the filter parity tests


def _ref(t, width, height, depth):
    return DataRef(t.data_ptr(), width, height, depth, width)


def _run(fn, src, dst, H):
    d, h, w = src.shape
    return fn(C.byref(_ref(src, w, h, d)), C.byref(_ref(dst, w, h, d)), C.byref(_ref(H, H.numel(), 1, 1)))


def _filter_both(nu, nv, views, seed):
    import torch

    p = F.config("c1")
    p.nu, p.nv = nu, nv
    H = torch.from_numpy(p.fft_kernel_real_f32).cuda()
    rng = np.random.default_rng(seed)
    src = torch.from_numpy((rng.standard_normal((views, nv, nu)) * 10).astype(np.float32)).cuda()
    want = torch.empty_like(src)
    got = torch.empty_like(src)
    assert _run(lib().fdk_filter_row_real32, src, want, H) == 0
    assert _run(lib().fdk_filter_row_real32_noalloc, src, got, H) == 0, lib().fdk_last_error()
    torch.cuda.synchronize()
    return got.cpu().numpy(), want.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    for nu, nv, views, seed in ((2048, 24, 3, 1), (256, 100, 4, 2)):  # W = 4096, then W = 512
        got, want = _filter_both(nu, nv, views, seed)
        err = float(np.abs(got - want).max() / np.abs(want).max())
        assert err <= TOL, (nu, err)


def test_noalloc_matches_the_fp64_oracle_at_w4096():
    import torch

    from oracle import oracle as O

    p = F.config("c1")
    p.nu, p.nv = 2048, 16  # W = 4096, the largest table the static array holds
    H = p.fft_kernel_real
    rng = np.random.default_rng(11)
    views = (rng.standard_normal((2, p.nv, p.nu)) * 10).astype(np.float32)
    src = torch.from_numpy(views).cuda()
    got = torch.empty_like(src)
    Hd = torch.from_numpy(H.astype(np.float32)).cuda()
    assert _run(lib().fdk_filter_row_real32_noalloc, src, got, Hd) == 0, lib().fdk_last_error()
    torch.cuda.synchronize()
    want = np.stack([O.filter_view(v, H, None, pad_n=3) for v in views])
    err = float(np.abs(got.cpu().numpy() - want).max() / np.abs(want).max())
    assert err <= TOL, err


def test_noalloc_rejects_filters_longer_than_the_static_tables():
    import torch

    src = torch.zeros((1, 4, 4100), dtype=torch.float32, device="cuda")
    dst = torch.zeros_like(src)
    H = torch.zeros(8192, dtype=torch.float32, device="cuda")
    rc = _run(lib().fdk_filter_row_real32_noalloc, src, dst, H)
    assert rc == -1 and b"no-allocation limit of 4096" in lib().fdk_last_error()
