"""Learned residual row filter for sparse-view, low-dose FDK (no reference counterpart).

Data (BASELINE C5): 256^3 volume of 1 mm voxels, 90 views over 360 deg of a 256^2 detector of
1.5 mm pixels, SOD 1000 / SID 1500 mm.  Phantoms: seeded random ellipsoids (10-30 per sample,
the benchmark distributions), sampled on the voxel grid and projected by the project's
ray-marching forward projector (fdk_forward_project); transmission noise Poisson(I0 exp(-mu p))
with I0 = 1e4 photons per ray, then -log(counts / I0) / mu.  The densities are read as relative
attenuation with mu = 0.02 / mm per unit density (water); the benchmark leaves mu unspecified.

Training: y = x + net(x) on every cosine-weighted, Hann-ramp-filtered detector row x; the rows go
to the staged FP32 backprojection; loss = volume MSE against the phantom; the gradient returns
through the exact backprojection adjoint (fdk_bp_adjoint) and the network's backward kernel;
Adam (lr 1e-3, cosine-decayed to 1e-5 over the run by default).  Every kernel is this library's
own (learn.cu, fproj.cu, filter.cu, bp_tma.cuh).

Plain Hann-ramp FDK (zero residual) is the fallback and the referee: on each held-out scan the
learned reconstruction is kept only when its error against the phantom is lower.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import time

import numpy as np

from . import _lib
from ._lib import LAYOUT_MIRROR, check, lib
from .backprojection import BackProjectionFDK, BoxT
from .filter import FilterEngine
from .geometry import config
from .phantom import random_ellipsoids

MU = 0.02   # 1/mm per unit density
I0 = 1.0e4  # photons per ray


def n_params() -> int:
    return lib().fdk_nn_param_count()


def init_params(seed: int = 0) -> np.ndarray:
    """He-style init for layers 1-2; zero last layer, so the untrained filter is plain FDK."""
    rng = np.random.default_rng(seed)
    w1 = rng.standard_normal(32 * 9) * np.sqrt(2.0 / 9)
    b1 = np.zeros(32)
    w2 = rng.standard_normal(32 * 32 * 9) * np.sqrt(2.0 / (32 * 9))
    b2 = np.zeros(32)
    w3 = np.zeros(32 * 9)
    b3 = np.zeros(1)
    p = np.concatenate([w1, b1, w2, b2, w3, b3]).astype(np.float32)
    assert p.size == n_params()
    return p


class Pipeline:
    """Device buffers and kernels for one scan geometry (torch for device memory only).

    input_window: the ramp-filter window of the rows the network reads ("hann", the geometry's
    own, or e.g. "ram-lak" to let the network learn its own apodization).  Plain FDK, the
    fallback and referee, always uses the geometry's window."""

    def __init__(self, param=None, device: int = 0, input_window: str | None = None):
        import torch

        self.torch = torch
        self.p = param or config("c5")
        p = self.p
        self.dev = torch.device("cuda", device)
        self.g = p.to_c()
        self.nviews = p.nProj
        self.rows = p.nProj * p.nv
        self.scale = float(1.0 / (p.SOD * p.SOD * p.AngularAndrampFactor))  # rows -> line-integral units
        t = lambda *shape: torch.empty(shape, dtype=torch.float32, device=self.dev)  # noqa: E731
        self.truth = t(p.nz, p.ny, p.nx)
        self.proj = t(p.nProj, p.nv, p.nu)
        self.y = t(p.nProj, p.nv, p.nu)
        self.grad = t(p.nProj, p.nv, p.nu)
        self.mirror = t(p.nProj, p.nu, p.nv, 2)
        self.res = t(p.nz, p.ny, p.nx)
        self.dparams = t(n_params())
        self.mats_h = p.proj_matrices()
        self.mats_d = torch.from_numpy(self.mats_h.reshape(-1)).to(self.dev)
        self.engine = FilterEngine(p.cos_sigma, p.fft_kernel_real_f32, pad_edge=4, device=device)
        self.input_window = input_window or p.str_filter
        if self.input_window != p.str_filter:
            q = dataclasses.replace(p, str_filter=self.input_window)
            self.engine_in = FilterEngine(p.cos_sigma, q.fft_kernel_real_f32, pad_edge=4, device=device)
        else:
            self.engine_in = self.engine
        self.bp = BackProjectionFDK(p.nv, p.nu, 128, p.nx, p.ny, p.nz, BoxT(0, 0, 0, p.nx, p.ny, p.nz // 2),
                                    BoxT(0, 0, p.nz // 2, p.nx, p.ny, p.nz // 2), "fp32", device)

    # ------------------------------------------------------------------ data
    def scan(self, seed: int, out_rows, plain_rows=None) -> np.ndarray:
        """Phantom `seed`: truth -> self.truth, the noisy views filtered with the input window ->
        out_rows, and with the geometry's window -> plain_rows (if given).  Returns ellipsoids."""
        p = self.p
        rng = np.random.default_rng(seed)
        ell = random_ellipsoids(seed, int(rng.integers(10, 31)), 0.5 * p.nx * p.dx)
        e = np.ascontiguousarray(ell, np.float64)
        check(lib().fdk_voxelize(C.byref(self.g), e.ctypes.data, len(e), self.truth.data_ptr(), None))
        check(lib().fdk_forward_project(C.byref(self.g), self.truth.data_ptr(), 0, p.nProj, self.proj.data_ptr(),
                                        None))
        check(lib().fdk_transmission_noise(self.proj.data_ptr(), self.proj.numel(), I0, MU,
                                           np.uint64(seed * 7919 + 17), None))
        self.engine_in.run_device(self.proj.data_ptr(), out_rows.data_ptr(), p.nProj, _lib.LAYOUT_ROWS,
                                  _lib.DTYPE_F32)
        if plain_rows is not None:
            self.engine.run_device(self.proj.data_ptr(), plain_rows.data_ptr(), p.nProj, _lib.LAYOUT_ROWS,
                                   _lib.DTYPE_F32)
        return ell

    def truth_of(self, seed: int):
        p = self.p
        rng = np.random.default_rng(seed)
        ell = random_ellipsoids(seed, int(rng.integers(10, 31)), 0.5 * p.nx * p.dx)
        e = np.ascontiguousarray(ell, np.float64)
        check(lib().fdk_voxelize(C.byref(self.g), e.ctypes.data, len(e), self.truth.data_ptr(), None))

    # ------------------------------------------------------------------ forward / loss / backward
    def reconstruct(self, params_d, x_rows) -> None:
        p = self.p
        if params_d is None:
            src = x_rows
        else:
            check(lib().fdk_nn_forward(params_d.data_ptr(), x_rows.data_ptr(), self.y.data_ptr(), self.rows, p.nu,
                                       self.scale, None))
            src = self.y
        check(lib().fdk_rows_to_mirror(src.data_ptr(), self.mirror.data_ptr(), p.nProj, p.nu, p.nv, None))
        self.bp.reset()
        self.bp.BP_device(self.mirror.data_ptr(), LAYOUT_MIRROR, self.mats_h, p.nProj)

    def fov_mask(self):
        """Voxels whose centre projects inside [0, nu-1) x [0, nv-1) in every view: the fully
        sampled field of view (a cylinder capped by the cone).  Bool tensor [z][y][x], cached."""
        if getattr(self, "_fov", None) is None:
            torch, p = self.torch, self.p
            z, y, x = torch.meshgrid(*(torch.arange(n, dtype=torch.float64, device=self.dev)
                                       for n in (p.nz, p.ny, p.nx)), indexing="ij")
            fov = torch.ones((p.nz, p.ny, p.nx), dtype=torch.bool, device=self.dev)
            for m in np.asarray(p.proj_matrices(np.float64)).reshape(-1, 12):
                w = m[8] * x + m[9] * y + m[10] * z + m[11]
                u = (m[0] * x + m[1] * y + m[2] * z + m[3]) / w
                v = (m[4] * x + m[5] * y + m[6] * z + m[7]) / w
                fov &= (w > 0) & (u >= 0) & (u < p.nu - 1) & (v >= 0) & (v < p.nv - 1)
            self._fov = fov
        return self._fov

    def mse_fov(self) -> float:
        """After mse(with_grad=True): the MSE over fov_mask() (the residual holds 2 d / N)."""
        p = self.p
        d = self.res * (0.5 * p.nx * p.ny * p.nz)
        return float((d[self.fov_mask()] ** 2).mean())

    def mse(self, with_grad: bool) -> float:
        p = self.p
        vol, _ = self.bp.volume_device()
        sse = C.c_double(0)
        check(lib().fdk_volume_mse(vol, self.truth.data_ptr(), self.res.data_ptr() if with_grad else None, p.nx, p.ny,
                                   p.nz, C.byref(sse), None))
        return sse.value / (p.nx * p.ny * p.nz)

    def gradient(self, params_d, x_rows, fov_only: bool = False) -> None:
        """After reconstruct() + mse(with_grad=True): parameter gradient into self.dparams.
        fov_only: the gradient of the MSE over the fully sampled field of view alone (the
        residual outside fov_mask() is zeroed before the adjoint)."""
        p = self.p
        if fov_only:
            self.res.mul_(self.fov_mask())
        self.grad.zero_()
        check(lib().fdk_bp_adjoint(C.byref(self.g), self.res.data_ptr(), self.mats_d.data_ptr(), p.nProj,
                                   self.grad.data_ptr(), None))
        check(lib().fdk_nn_backward(params_d.data_ptr(), x_rows.data_ptr(), self.grad.data_ptr(),
                                    self.dparams.data_ptr(), self.rows, p.nu, self.scale, None))


def train(n_train: int = 2000, epochs: int = 20, lr: float = 1e-3, seed0: int = 1000, params=None, log=print,
          time_limit_s: float | None = None, on_epoch=None, schedule: str = "constant",
          input_window: str | None = None, batch: int = 1, loss_region: str = "volume") -> dict:
    """Adam on volume MSE; the training scans are generated once.  batch: phantoms per Adam
    step (their gradients averaged; 1 = one phantom per step).  loss_region: "volume" (the
    whole cube) or "fov" (the fully sampled field of view, Pipeline.fov_mask).
    schedule: "constant" (lr throughout) or "cosine" (lr decayed to lr/100 over all steps).
    on_epoch(epoch, params, history), when given, runs after every epoch (checkpointing)."""
    import torch

    pl = Pipeline(input_window=input_window)
    p = pl.p
    xs = torch.empty((n_train, p.nProj, p.nv, p.nu), dtype=torch.float32, device=pl.dev)
    t0 = time.time()
    for i in range(n_train):
        pl.scan(seed0 + i, xs[i])
    torch.cuda.synchronize()
    log(f"generated {n_train} training scans in {time.time() - t0:.1f} s")
    w = torch.from_numpy(init_params() if params is None else np.asarray(params, np.float32)).to(pl.dev)
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    gsum = torch.zeros_like(w)
    hist, step, t0 = [], 0, time.time()
    total = max(1, (n_train // batch) * epochs)
    rng = np.random.default_rng(7)
    stopped = False
    for ep in range(epochs):
        order = rng.permutation(n_train)
        tot = 0.0
        n_done = 0
        for b0 in range(0, n_train - batch + 1, batch):
            for i in order[b0:b0 + batch]:
                pl.truth_of(seed0 + int(i))
                pl.reconstruct(w, xs[i])
                tot += pl.mse(with_grad=True)
                pl.gradient(w, xs[i], fov_only=loss_region == "fov")
                if batch > 1:
                    gsum += pl.dparams
            n_done += batch
            step += 1
            if batch > 1:
                torch.mul(gsum, 1.0 / batch, out=pl.dparams)
                gsum.zero_()
            lr_t = lr if schedule == "constant" else lr * (0.01 + 0.99 * 0.5 * (1 + math.cos(math.pi * step / total)))
            check(lib().fdk_adam_step(w.data_ptr(), pl.dparams.data_ptr(), m.data_ptr(), v.data_ptr(), w.numel(),
                                      lr_t, 0.9, 0.999, 1e-8, step, None))
            if time_limit_s is not None and time.time() - t0 > time_limit_s:
                stopped = True
                break
        torch.cuda.synchronize()
        hist.append(tot / max(1, n_done))
        log(f"epoch {ep}: train MSE {hist[-1]:.4e} ({time.time() - t0:.0f} s, {step} steps)")
        if on_epoch is not None:
            on_epoch(ep, w.cpu().numpy(), list(hist))
        if stopped:
            break
    return {"params": w.cpu().numpy(), "history": hist, "steps": step, "seconds": time.time() - t0,
            "epochs_completed": len(hist) if not stopped else len(hist) - 1, "stopped_early": stopped}


def evaluate(params, n_test: int = 200, seed0: int = 5000, input_window: str | None = None) -> dict:
    """Held-out scans: MSE of plain FDK, of the learned filter, and of the gated choice, over the
    whole volume and over the fully sampled field of view (Pipeline.fov_mask)."""
    import torch

    pl = Pipeline(input_window=input_window)
    p = pl.p
    x = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device=pl.dev)
    xp = torch.empty_like(x) if pl.engine_in is not pl.engine else x
    w = torch.from_numpy(np.asarray(params, np.float32)).to(pl.dev)
    plain, learned, kept, plain_f, learned_f = [], [], [], [], []
    for i in range(n_test):
        pl.scan(seed0 + i, x, xp if xp is not x else None)
        pl.reconstruct(None, xp)
        e0 = pl.mse(with_grad=True)
        plain_f.append(pl.mse_fov())
        pl.reconstruct(w, x)
        e1 = pl.mse(with_grad=True)
        learned_f.append(pl.mse_fov())
        plain.append(e0)
        learned.append(e1)
        kept.append(min(e0, e1))
    plain, learned, kept, plain_f, learned_f = map(np.asarray, (plain, learned, kept, plain_f, learned_f))
    kept_f = np.where(learned < plain, learned_f, plain_f)  # the gate decides on the whole volume
    return {"n": n_test, "mse_plain": float(plain.mean()), "mse_learned": float(learned.mean()),
            "mse_kept": float(kept.mean()), "learned_better_frac": float((learned < plain).mean()),
            "mse_reduction": float(1 - kept.mean() / plain.mean()),
            "rmse_reduction": float(1 - np.sqrt(kept).mean() / np.sqrt(plain).mean()),
            "fov_fraction": float(pl.fov_mask().float().mean()),
            "fov_mse_plain": float(plain_f.mean()), "fov_mse_kept": float(kept_f.mean()),
            "fov_mse_reduction": float(1 - kept_f.mean() / plain_f.mean())}
