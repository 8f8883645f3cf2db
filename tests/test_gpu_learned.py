"""Learned residual filter: the projector against the oracle, the exact backprojection adjoint
(dot-product test), the network kernels against the CPU oracle (whose own gradients are checked by
finite differences in tests/test_nn_oracle.py), the whole gradient by finite differences, a short
training that must beat plain FDK, and the committed trained network on held-out scans."""
import ctypes as C
import os

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200 import learned as Lr
from fdk_b200._lib import check, lib
from oracle import nn_oracle as N
from oracle import oracle as O
from tests.helpers import small_param

pytestmark = pytest.mark.gpu


def test_forward_projector_vs_oracle():
    import torch

    from fdk_b200.phantom import phantom_for

    p = small_param(48, 56, 40, 6)
    ell = phantom_for(p, 4, 12)
    vol = O.ellipsoid_volume(ell, p)
    d_vol = torch.from_numpy(vol).cuda()
    out = torch.empty((6, p.nv, p.nu), dtype=torch.float32, device="cuda")
    g = p.to_c()
    check(lib().fdk_forward_project(C.byref(g), d_vol.data_ptr(), 0, 6, out.data_ptr(), None))
    torch.cuda.synchronize()
    want = np.stack([O.forward_project(vol, p, a) for a in O.view_angles(p)])
    got = out.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-4
    if os.path.exists(os.path.join(O.REF_DIR, "libref_cpu.so")):
        # and against the reference's own 3dct ForwardProjection (3dct/3dct.cpp:430-573)
        ref = np.stack([O.RefCPU().forward_projection(vol, p, i) for i in range(6)])
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-4


def test_bp_adjoint_dot_product():
    """<BP(p), r> == <p, BP^T(r)> for the staged FP32 backprojection and its adjoint kernel."""
    import torch

    n, views = 40, 12
    p = small_param(n, 48, 44, views)
    rng = np.random.default_rng(0)
    rows = torch.from_numpy(rng.standard_normal((views, p.nv, p.nu)).astype(np.float32)).cuda()
    r = torch.from_numpy(rng.standard_normal((n, n, n)).astype(np.float32)).cuda()  # [z][y][x]
    mirror = torch.empty((views, p.nu, p.nv, 2), dtype=torch.float32, device="cuda")
    check(lib().fdk_rows_to_mirror(rows.data_ptr(), mirror.data_ptr(), views, p.nu, p.nv, None))
    bp = F.BackProjectionFDK(p.nv, p.nu, 32, n, n, n, F.BoxT(0, 0, 0, n, n, n // 2), F.BoxT(0, 0, n // 2, n, n, n // 2),
                             "fp32")
    mats = p.proj_matrices()
    bp.BP_device(mirror.data_ptr(), F.LAYOUT_MIRROR, mats, views)
    vol = bp.GetVolumeData()  # [z][y][x] for the full slab pair
    a = float((vol.astype(np.float64) * r.cpu().numpy().astype(np.float64)).sum())
    grad = torch.zeros_like(rows)
    d_mats = torch.from_numpy(mats.reshape(-1)).cuda()
    g = p.to_c()
    check(lib().fdk_bp_adjoint(C.byref(g), r.data_ptr(), d_mats.data_ptr(), views, grad.data_ptr(), None))
    torch.cuda.synchronize()
    b = float((rows.double() * grad.double()).sum())
    assert abs(a - b) <= 1e-4 * abs(a), (a, b)


def test_network_kernels_vs_cpu_oracle():
    import torch

    rng = np.random.default_rng(1)
    rows, L, s = 37, 64, 0.25
    params = (rng.standard_normal(N.NPARAM) * 0.2).astype(np.float32)
    x = rng.standard_normal((rows, L)).astype(np.float32) * 4
    dy = rng.standard_normal((rows, L)).astype(np.float32)
    dp, dx, ddy = (torch.from_numpy(a).cuda() for a in (params, x, dy))
    y = torch.empty_like(dx)
    g = torch.empty_like(dp)
    check(lib().fdk_nn_forward(dp.data_ptr(), dx.data_ptr(), y.data_ptr(), rows, L, s, None))
    check(lib().fdk_nn_backward(dp.data_ptr(), dx.data_ptr(), ddy.data_ptr(), g.data_ptr(), rows, L, s, None))
    torch.cuda.synchronize()
    y_ref, _ = N.forward(params, x, s, round_bf16=True)
    g_ref = N.backward(params, x, dy, s, round_bf16=True)
    assert np.abs(y.cpu().numpy() - y_ref).max() <= 2e-2 * np.abs(y_ref).max()
    rel = np.linalg.norm(g.cpu().numpy() - g_ref) / np.linalg.norm(g_ref)
    assert rel <= 2e-2, rel
    assert Lr.n_params() == N.NPARAM


def test_end_to_end_gradient_finite_difference():
    """Directional derivative of the volume MSE along the last layer (W3, b3), where the loss is
    exactly quadratic in the step, from the gradient kernels (backprojection adjoint + network
    backward) against a central difference through the forward pipeline (network + BP + MSE)."""
    import torch

    p = small_param(40, 40, 40, 24)
    pl = Lr.Pipeline(p)
    x = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device="cuda")
    pl.scan(7, x)
    rng = np.random.default_rng(3)
    w0 = Lr.init_params()
    k_w3 = N.NPARAM - 32 * 9 - 1
    w0[k_w3:] = (rng.standard_normal(32 * 9 + 1) * 0.05).astype(np.float32)
    d = np.zeros_like(w0)
    d[k_w3:] = rng.standard_normal(32 * 9 + 1).astype(np.float32)

    def loss(w_host, grad=False):
        w = torch.from_numpy(w_host).cuda()
        pl.truth_of(7)
        pl.reconstruct(w, x)
        e = pl.mse(grad)
        if grad:
            pl.gradient(w, x)
            torch.cuda.synchronize()
            return e, pl.dparams.cpu().numpy().astype(np.float64)
        return e

    l0, g = loss(w0, grad=True)
    t = 0.05 * l0 / abs(float(g @ d))
    wp, wm = (w0 + t * d).astype(np.float32), (w0 - t * d).astype(np.float32)
    predicted = float(g @ (wp.astype(np.float64) - wm))
    measured = loss(wp) - loss(wm)
    assert abs(measured - predicted) <= 1e-2 * abs(predicted), (measured, predicted)


def test_short_training_beats_plain_fdk():
    """A few Adam steps on a handful of small noisy scans already lower the volume error below the
    plain Hann-ramp reconstruction of the same scans."""
    import torch

    p = small_param(48, 48, 48, 30)
    pl = Lr.Pipeline(p)
    xs = torch.empty((4, p.nProj, p.nv, p.nu), dtype=torch.float32, device="cuda")
    for i in range(4):
        pl.scan(100 + i, xs[i])
    w = torch.from_numpy(Lr.init_params()).cuda()
    m, v = torch.zeros_like(w), torch.zeros_like(w)
    plain = []
    for i in range(4):
        pl.truth_of(100 + i)
        pl.reconstruct(None, xs[i])
        plain.append(pl.mse(False))
    step = 0
    for ep in range(15):
        for i in range(4):
            pl.truth_of(100 + i)
            pl.reconstruct(w, xs[i])
            pl.mse(True)
            pl.gradient(w, xs[i])
            step += 1
            check(lib().fdk_adam_step(w.data_ptr(), pl.dparams.data_ptr(), m.data_ptr(), v.data_ptr(), w.numel(), 1e-3,
                                      0.9, 0.999, 1e-8, step, None))
    learned = []
    for i in range(4):
        pl.truth_of(100 + i)
        pl.reconstruct(w, xs[i])
        learned.append(pl.mse(False))
    assert np.mean(learned) < 0.97 * np.mean(plain), (np.mean(learned), np.mean(plain))


def test_trained_weights_beat_plain_fdk_on_held_out_scans():
    """The committed C5 network (fdk_b200/weights/residual_c5.npz) against plain Hann-ramp FDK on
    held-out phantoms (seeds outside the training range): lower volume MSE on every scan and a
    clear mean gain.  The full 200-scan evaluation is fdk_b200.train_learned's output."""
    import os

    path = os.path.join(os.path.dirname(Lr.__file__), "weights", "residual_c5.npz")
    d = np.load(path)
    window = str(d["input_window"]) if "input_window" in d.files else None
    ev = Lr.evaluate(d["params"], n_test=8, seed0=5000, input_window=window)
    print(ev)
    assert ev["learned_better_frac"] == 1.0
    assert ev["mse_reduction"] >= 0.10, ev


def test_field_of_view_weights_beat_plain_fdk_inside_the_field_of_view():
    """The C5 network trained on the loss over the fully sampled field of view
    (fdk_b200/weights/residual_c5_fov.npz, `train_learned --loss-region fov`) against plain FDK
    on held-out phantoms: lower MSE on every scan, and inside the field of view a larger cut than
    the volume-trained weights give there (the 200-scan figures are in residual_c5_fov.json)."""
    import os

    path = os.path.join(os.path.dirname(Lr.__file__), "weights", "residual_c5_fov.npz")
    d = np.load(path)
    ev = Lr.evaluate(d["params"], n_test=8, seed0=5000)
    print(ev)
    assert ev["learned_better_frac"] == 1.0
    assert ev["fov_mse_reduction"] >= 0.17, ev
