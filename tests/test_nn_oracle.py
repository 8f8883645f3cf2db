"""The CPU oracle of the learned filter: analytic gradients against central finite differences
(float64, no BF16 rounding), so that the GPU kernels are compared with a checked reference."""
import numpy as np

from oracle import nn_oracle as N


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(N.NPARAM) * 0.1
    x = rng.standard_normal((3, 20))
    dy = rng.standard_normal((3, 20))
    s = 0.7
    g = N.backward(p, x, dy, s, round_bf16=False)
    idx = rng.choice(N.NPARAM, 60, replace=False)
    eps = 1e-6
    fd = []
    for i in idx:
        pp = p.copy()
        pp[i] += eps
        yp, _ = N.forward(pp, x, s, False)
        pm = p.copy()
        pm[i] -= eps
        ym, _ = N.forward(pm, x, s, False)
        fd.append(((yp - ym) * dy).sum() / (2 * eps))
    assert np.abs(np.array(fd) - g[idx]).max() <= 1e-6 * np.abs(g[idx]).max()


def test_zero_last_layer_is_identity():
    from fdk_b200 import learned

    p = learned.init_params()
    x = np.random.default_rng(1).standard_normal((4, 32))
    y, _ = N.forward(p, x, 0.5)
    assert np.array_equal(y, x.astype(np.float64))
