"""The filter matrix of the tensor-core filter: applied to cosine-weighted rows in FP64 it must
reproduce the FFT filter (pads, circular kernel, crop) of the FP64 oracle."""
import numpy as np
import pytest

import fdk_b200 as F
from oracle import oracle as O
from tests.helpers import small_param


@pytest.mark.parametrize("nu,pad", [(256, 4), (200, 3), (1536, 4)])
def test_matrix_reproduces_fft_filter(nu, pad):
    p = small_param(64, nu, 6, 2)
    H = O.filter_design(p.str_filter, p.nu)
    cos = O.cos_table(p)
    rng = np.random.default_rng(nu)
    view = (rng.standard_normal((6, nu)) * 30 + 50).astype(np.float32)
    want = O.filter_view(view, H, cos, pad_n=pad, transpose=False).astype(np.float64)
    M = F.toeplitz_matrix(H, nu, pad)
    got = (view.astype(np.float64) * cos.astype(np.float64)) @ M.T
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
