"""Python access to the CPU oracle and to the reference's own compiled code.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` -- as the checker, never as the thing measured or
shipped.  The product package (``fdk_b200``) never imports this module.

* ``liboracle.so`` (built from ``fdk_oracle.c`` by ``oracle/Makefile``): the C
  restatement of the reference's geometry, ramp filter and backprojection, with a
  bit-level emulation of the reference kernel's ``mad.rz.ftz`` arithmetic and an
  FP64 variant.
* ``_ref/libref_cpu.so`` (built by ``oracle/build_ref.sh`` from the reference's own
  sources): ``Parameter::init``, ``filterImageRow`` and the 3dct CPU FDK.
* ``_ref/libref_gpu_bp.so`` / ``_ref/libref_gpu_filter.so``: the reference's own
  ``cudaFdkBP`` kernel and cuFFT filter plugin, compiled for sm_100a (GPU only).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

FILTERS = {"none": 0, "ram-lak": 1, "shepp-logan": 2, "cosine": 3, "hamming": 4, "hann": 5}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_lp6 = C.c_long * 6

_lib = None


def lib():
    """Load liboracle.so (building it with make if it is missing)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess

            subprocess.check_call(["make", "-s", "-C", HERE])
        L = C.CDLL(path)
        L.orc_nextpow2.restype = C.c_int
        L.orc_filter_design.argtypes = [C.c_int, C.c_int, C.c_int, _f64p]
        L.orc_filter_design.restype = C.c_int
        L.orc_angular_ramp_factor.argtypes = [C.c_double, C.c_long, C.c_double, C.c_double]
        L.orc_angular_ramp_factor.restype = C.c_double
        L.orc_cos_table.argtypes = [C.c_long, C.c_long] + [C.c_double] * 7 + [_f32p]
        L.orc_proj_matrix.argtypes = ([C.c_long] * 3 + [C.c_double] * 3 + [C.c_long] * 2 +
                                      [C.c_double] * 5 + [_f64p])
        L.orc_filter_view.argtypes = [_f32p, _f32p, C.c_long, C.c_long, C.c_void_p, _f64p,
                                      C.c_int, C.c_int, C.c_int]
        L.orc_filter_view.restype = C.c_int
        L.orc_fma_rz.argtypes = [C.c_float] * 3
        L.orc_fma_rz.restype = C.c_float
        L.orc_bp_ref32.argtypes = [_f32p, _lp6, C.c_long, C.c_long, _f32p, C.c_int, C.c_int,
                                   _f32p, C.c_int]
        L.orc_bp_f64.argtypes = [_f64p, _lp6, C.c_long, C.c_long, _f32p, C.c_int, C.c_int,
                                 _f64p, C.c_int]
        L.orc_transform_volume.argtypes = [_f32p, _f32p, C.c_long, C.c_long, C.c_long]
        L.orc_rtk_bp.argtypes = [C.c_int * 3, C.c_int * 3, _f32p, _f32p, _f32p, _f32p]
        L.orc_ellipsoid_projection.argtypes = [_f64p, C.c_int, C.c_long, C.c_long, C.c_double,
                                               C.c_double, C.c_double, C.c_double, C.c_double, _f32p]
        L.orc_ellipsoid_volume.argtypes = [_f64p, C.c_int, C.c_long, C.c_long, C.c_long,
                                           C.c_double, C.c_double, C.c_double, _f32p]
        L.orc_forward_project.argtypes = ([_f32p] + [C.c_long] * 3 + [C.c_float] * 3 + [C.c_long] * 2 +
                                          [C.c_float] * 4 + [C.c_double, _f32p])
        L.orc_fdk_sampled.argtypes = [_f32p, C.c_int, C.c_long, C.c_long, C.c_void_p, _f64p, C.c_int, C.c_int,
                                      _f64p, np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS"), C.c_long,
                                      _f64p, C.c_void_p]
        L.orc_fdk_sampled.restype = C.c_int
        _lib = L
    return _lib


# --------------------------------------------------------------------------- geometry
def nextpow2(n: int) -> int:
    return lib().orc_nextpow2(int(n))


def filter_design(ftype: str, nu: int, d: int = 1) -> np.ndarray:
    W = nextpow2(nu)
    out = np.zeros(W, np.float64)
    r = lib().orc_filter_design(FILTERS[ftype], int(nu), int(d), out)
    assert r == W
    return out


def angular_ramp_factor(g) -> float:
    return lib().orc_angular_ramp_factor(g.du, g.nProj, g.SID, g.SOD)


def cos_table(g) -> np.ndarray:
    out = np.zeros((g.nv, g.nu), np.float32)
    lib().orc_cos_table(g.nu, g.nv, g.du, g.dv, g.offset_nu, g.offset_nv, g.SID, g.SOD,
                        angular_ramp_factor(g), out)
    return out


def view_angles(g) -> np.ndarray:
    """direction * deg / 180 * PI + volume_postion_angle (common/type.h:4729, 4824)."""
    deg = np.arange(g.nProj, dtype=np.float64) * g.scan_angle / float(g.nProj)
    return g.direction * deg / 180.0 * np.pi + g.volume_postion_angle


def proj_matrices(g) -> np.ndarray:
    """FP64 3x4 matrices (n, 12), CalculateProjMat (common/type.h:4898-4944)."""
    out = np.zeros((g.nProj, 12), np.float64)
    tmp = np.zeros(12, np.float64)
    for i, a in enumerate(view_angles(g)):
        lib().orc_proj_matrix(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.nu, g.nv, g.du, g.dv,
                              g.SID, g.SOD, float(a), tmp)
        out[i] = tmp
    return out


# --------------------------------------------------------------------------- filter
def filter_view(src: np.ndarray, H: np.ndarray, cos_tab=None, pad_n: int = 4,
                transpose: bool = False) -> np.ndarray:
    """Row filter of one view (nv, nu) in FP64 arithmetic; FilterLib.h:8-196."""
    src = np.ascontiguousarray(src, np.float32)
    nv, nu = src.shape
    dst = np.zeros((nu, nv) if transpose else (nv, nu), np.float32)
    cp = None
    if cos_tab is not None:
        cos_tab = np.ascontiguousarray(cos_tab, np.float32)
        cp = cos_tab.ctypes.data
    r = lib().orc_filter_view(src, dst, nu, nv, cp, np.ascontiguousarray(H, np.float64),
                              len(H), pad_n, int(transpose))
    assert r == 0
    return dst


# --------------------------------------------------------------------------- backprojection
def bp_ref32(vol: np.ndarray, top, depth_bottom: int, nz: int, proj: np.ndarray,
             mats: np.ndarray) -> None:
    """cudaFdkBP<1,false,sym> emulated bit for bit (in place on vol, [x][y][zs])."""
    n, height, width = proj.shape
    lib().orc_bp_ref32(vol, _lp6(*top), depth_bottom, nz, np.ascontiguousarray(proj, np.float32),
                       width, height, np.ascontiguousarray(mats, np.float32).reshape(-1), n)


def bp_f64(vol: np.ndarray, top, depth_bottom: int, nz: int, proj: np.ndarray,
           mats: np.ndarray) -> None:
    n, height, width = proj.shape
    lib().orc_bp_f64(vol, _lp6(*top), depth_bottom, nz, np.ascontiguousarray(proj, np.float32),
                     width, height, np.ascontiguousarray(mats, np.float64).reshape(-1), n)


class SampledFDK:
    """FP64 FDK at a fixed list of voxels (orc_fdk_sampled), fed views in any number of calls.

    vox: (n, 3) int array of voxel indices (x, y, z).  add(views, first) filters the raw views
    first .. first+len(views)-1 (FP32, (n, nv, nu)) in double and accumulates their samples;
    values holds the FP64 reconstruction at the voxels, edge marks the knife-edge voxels."""

    def __init__(self, g, vox: np.ndarray, pad_n: int = 4):
        self.g = g
        self.vox = np.ascontiguousarray(vox, np.int32).reshape(-1, 3)
        self.values = np.zeros(len(self.vox), np.float64)
        self.edge = np.zeros(len(self.vox), np.uint8)
        self.H = filter_design(g.str_filter, g.nu)
        self.cos = cos_table(g)
        self.mats = proj_matrices(g)
        self.pad_n = pad_n

    def add(self, views: np.ndarray, first: int) -> None:
        views = np.ascontiguousarray(views, np.float32)
        n = views.shape[0]
        mats = np.ascontiguousarray(self.mats[first:first + n])
        r = lib().orc_fdk_sampled(views.reshape(-1), n, self.g.nu, self.g.nv, self.cos.ctypes.data, self.H,
                                  len(self.H), self.pad_n, mats.reshape(-1), self.vox.reshape(-1), len(self.vox),
                                  self.values, self.edge.ctypes.data)
        assert r == 0, r


def sample_voxels(nx: int, ny: int, nz: int, n_random: int, seed: int, slices: bool = True) -> np.ndarray:
    """Voxel list for a sampled check: n_random seeded uniform voxels, plus (slices) every voxel
    of the central x, y and z slices.  (n, 3) int32 (x, y, z)."""
    rng = np.random.default_rng(seed)
    parts = [np.stack([rng.integers(0, nx, n_random), rng.integers(0, ny, n_random),
                       rng.integers(0, nz, n_random)], 1)]
    if slices:
        a, b = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
        parts.append(np.stack([np.full(a.size, nx // 2), a.ravel(), b.ravel()], 1))
        a, b = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        parts.append(np.stack([a.ravel(), np.full(a.size, ny // 2), b.ravel()], 1))
        a, b = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        parts.append(np.stack([a.ravel(), b.ravel(), np.full(a.size, nz // 2)], 1))
    return np.ascontiguousarray(np.concatenate(parts), np.int32)


def transform_volume(src: np.ndarray, nxs: int, nys: int, D: int) -> np.ndarray:
    dst = np.zeros(nxs * nys * D, np.float32)
    lib().orc_transform_volume(np.ascontiguousarray(src, np.float32).reshape(-1), dst, nxs, nys, D)
    return dst.reshape(D, nys, nxs)


def rtk_bp(proj: np.ndarray, mats: np.ndarray, vol_in: np.ndarray) -> np.ndarray:
    n, H, W = proj.shape
    nz, ny, nx = vol_in.shape
    out = np.zeros_like(vol_in, dtype=np.float32)
    lib().orc_rtk_bp((C.c_int * 3)(W, H, n), (C.c_int * 3)(nx, ny, nz),
                     np.ascontiguousarray(mats, np.float32).reshape(-1),
                     np.ascontiguousarray(vol_in, np.float32).reshape(-1),
                     out.reshape(-1), np.ascontiguousarray(proj, np.float32).reshape(-1))
    return out


# --------------------------------------------------------------------------- phantom
def ellipsoid_projection(ell: np.ndarray, g, angle: float) -> np.ndarray:
    out = np.zeros((g.nv, g.nu), np.float32)
    e = np.ascontiguousarray(ell, np.float64).reshape(-1)
    lib().orc_ellipsoid_projection(e, len(e) // 16, g.nu, g.nv, g.du, g.dv, g.SID, g.SOD,
                                   float(angle), out)
    return out


def ellipsoid_volume(ell: np.ndarray, g) -> np.ndarray:
    out = np.zeros((g.nz, g.ny, g.nx), np.float32)
    e = np.ascontiguousarray(ell, np.float64).reshape(-1)
    lib().orc_ellipsoid_volume(e, len(e) // 16, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, out)
    return out


def forward_project(vol: np.ndarray, g, angle: float) -> np.ndarray:
    """Ray-marching projector (genProj kernel_forwardProject semantics) of a [z][y][x] volume."""
    out = np.zeros((g.nv, g.nu), np.float32)
    lib().orc_forward_project(np.ascontiguousarray(vol, np.float32).reshape(-1), g.nx, g.ny, g.nz, g.dx, g.dy,
                              g.dz, g.nu, g.nv, g.du, g.dv, g.SID, g.SOD, float(angle), out)
    return out


# --------------------------------------------------------------------------- reference code
class RefCPU:
    """The reference's own CPU code (oracle/_ref/libref_cpu.so)."""

    def __init__(self):
        path = os.path.join(REF_DIR, "libref_cpu.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.refc_parameter.argtypes = ([C.c_long] * 3 + [C.c_double] * 3 + [C.c_long] * 2 +
                                     [C.c_double] * 6 + [C.c_long, C.c_double, C.c_long,
                                                         C.c_double, C.c_int, C.c_void_p, C.c_int,
                                                         C.c_void_p, C.c_void_p, C.c_void_p])
        L.refc_parameter.restype = C.c_int
        L.refc_filter_rows.argtypes = [_f64p, C.c_int, _f32p, _f32p, C.c_int, C.c_int]
        L.refc_cpu_fdk.argtypes = ([C.c_long] * 3 + [C.c_double] * 3 + [C.c_long] * 2 +
                                   [C.c_double] * 4 + [C.c_long, C.c_double, C.c_long, C.c_double,
                                                       C.c_int, _f32p, C.c_int, C.c_int, _f32p,
                                                       C.c_int])
        L.refc_fdk_create.restype = C.c_void_p
        L.refc_fdk_create.argtypes = ([C.c_long] * 3 + [C.c_double] * 3 + [C.c_long] * 2 +
                                      [C.c_double] * 4 + [C.c_long, C.c_double, C.c_long, C.c_double,
                                                          C.c_int])
        L.refc_fdk_run.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.refc_forward_projection.argtypes = ([C.c_long] * 3 + [C.c_double] * 3 + [C.c_long] * 2 +
                                              [C.c_double] * 4 + [C.c_long, C.c_double, C.c_long, C.c_double,
                                                                  _f32p, C.c_int, _f32p, C.c_int])
        L.refc_forward_projection.restype = C.c_int
        L.refc_fdk_destroy.argtypes = [C.c_void_p]
        self.L = L

    def forward_projection(self, vol: np.ndarray, g, view: int, threads: int = 0) -> np.ndarray:
        """3dct ForwardProjection<float> of a [z][y][x] volume for view `view`: (nv, nu)."""
        out = np.zeros((g.nv, g.nu), np.float32)
        r = self.L.refc_forward_projection(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.nu, g.nv, g.du, g.dv, g.SID, g.SOD,
                                           g.direction, g.scan_angle, g.nProj, g.volume_postion_angle,
                                           np.ascontiguousarray(vol, np.float32).reshape(-1), int(view),
                                           out.reshape(-1), int(threads))
        assert r == 0, r
        return out

    def fdk_handle(self, g, ftype="hann"):
        """Persistent reference CPU FDK (tables and buffers built once, outside timing)."""
        h = self.L.refc_fdk_create(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.nu, g.nv, g.du, g.dv, g.SID,
                                   g.SOD, g.direction, g.scan_angle, g.nProj, g.volume_postion_angle,
                                   FILTERS[ftype])
        assert h, "refc_fdk_create failed"
        return h

    def fdk_run(self, h, proj: np.ndarray, first: int, threads: int = 0) -> None:
        proj = np.ascontiguousarray(proj, np.float32)
        assert self.L.refc_fdk_run(h, proj.ctypes.data, int(first), int(proj.shape[0]), int(threads)) == 0

    def fdk_destroy(self, h) -> None:
        self.L.refc_fdk_destroy(h)

    def parameter(self, g, ftype="hann"):
        W = nextpow2(g.nu)
        H = np.zeros(W, np.float64)
        cos = np.zeros((g.nv, g.nu), np.float32)
        mats = np.zeros((g.nProj, 12), np.float32)
        aaf = C.c_double(0)
        r = self.L.refc_parameter(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.nu, g.nv, g.du, g.dv,
                                  g.offset_nu, g.offset_nv, g.SID, g.SOD, g.direction,
                                  g.scan_angle, g.nProj, g.volume_postion_angle, FILTERS[ftype],
                                  H.ctypes.data, W, cos.ctypes.data, mats.ctypes.data,
                                  C.addressof(aaf))
        assert r == W, r
        return dict(H=H, cos=cos, mats=mats, aaf=aaf.value)

    def filter_rows(self, H: np.ndarray, src: np.ndarray) -> np.ndarray:
        src = np.ascontiguousarray(src, np.float32)
        dst = np.zeros_like(src)
        h, w = src.shape
        assert self.L.refc_filter_rows(np.ascontiguousarray(H, np.float64), len(H), src, dst, w, h) == 0
        return dst

    def cpu_fdk(self, g, proj: np.ndarray, first: int, vol: np.ndarray, threads: int = 0,
                ftype="hann") -> None:
        proj = np.ascontiguousarray(proj, np.float32)
        r = self.L.refc_cpu_fdk(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.nu, g.nv, g.du, g.dv,
                                g.SID, g.SOD, g.direction, g.scan_angle, g.nProj,
                                g.volume_postion_angle, FILTERS[ftype], proj.reshape(-1),
                                int(first), int(proj.shape[0]), vol.reshape(-1), int(threads))
        assert r == 0, r


class RefGPU:
    """The reference's own GPU code compiled for sm_100a (needs a GPU)."""

    def __init__(self):
        bp = os.path.join(REF_DIR, "libref_gpu_bp.so")
        fl = os.path.join(REF_DIR, "libref_gpu_filter.so")
        self.bp = C.CDLL(bp)
        self.bp.refg_bp_create.restype = C.c_void_p
        self.bp.refg_bp_create.argtypes = [C.c_int] * 6 + [_lp6, _lp6]
        self.bp.refg_bp.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_int, C.c_int, _f32p, C.c_int]
        self.bp.refg_bp_get_volume.argtypes = [C.c_void_p, _f32p, C.c_long]
        self.bp.refg_bp_destroy.argtypes = [C.c_void_p]
        self.bp.refg_bp_kernel_ms.argtypes = [C.c_void_p, C.c_int, C.c_int]
        self.bp.refg_bp_kernel_ms.restype = C.c_float
        self.flt = C.CDLL(fl)
        self.flt.refg_filter.argtypes = [C.c_void_p] * 4 + [C.c_int] * 4

    def backproject(self, proj_batches, mats_batches, nx, ny, nz, top, bottom):
        """Run BackProjectionFDK over the batches; returns GetVolumeData's [zs][y][x]."""
        width, height = proj_batches[0].shape[2], proj_batches[0].shape[1]
        h = self.bp.refg_bp_create(width, height, 32, nx, ny, nz, _lp6(*top), _lp6(*bottom))
        assert h, "BackProjectionFDK construction failed"
        try:
            for p, m in zip(proj_batches, mats_batches):
                r = self.bp.refg_bp(h, 1, np.ascontiguousarray(p, np.float32).reshape(-1), width,
                                    height, np.ascontiguousarray(m, np.float32).reshape(-1),
                                    p.shape[0])
                assert r == 0, r
            D = top[5] + bottom[5]
            out = np.zeros(top[3] * top[4] * D, np.float32)
            assert self.bp.refg_bp_get_volume(h, out, out.size) == 0
            return out.reshape(D, top[4], top[3])
        finally:
            self.bp.refg_bp_destroy(h)

    def time_bp(self, proj: np.ndarray, mats: np.ndarray, nx, ny, nz, top, bottom, calls: int = 4,
                launches: int = 4) -> dict:
        """Speed of the reference's BackProjectionFDK on one GPU: `calls` stock BP(TRANSPOSE = 1)
        calls of the views (host, (n <= 32, nu, nv) transposed FP32; each call copies them to
        the device and synchronises, backprojectionFDK.cu:229-276), timed by the host clock,
        then `launches` launches of its kernel as BP() issues them, timed by CUDA events.
        Returns ms per call and per launch."""
        import time

        n, height, width = proj.shape
        proj = np.ascontiguousarray(proj, np.float32).reshape(-1)
        mats = np.ascontiguousarray(mats, np.float32).reshape(-1)
        h = self.bp.refg_bp_create(width, height, 32, nx, ny, nz, _lp6(*top), _lp6(*bottom))
        assert h, "BackProjectionFDK construction failed"
        try:
            assert self.bp.refg_bp(h, 1, proj, width, height, mats, n) == 0  # warm-up
            t0 = time.perf_counter()
            for _ in range(calls):
                assert self.bp.refg_bp(h, 1, proj, width, height, mats, n) == 0
            call_ms = 1e3 * (time.perf_counter() - t0) / calls
            kernel_ms = float(self.bp.refg_bp_kernel_ms(h, n, launches))
            assert kernel_ms > 0, kernel_ms
            return {"call_ms": call_ms, "kernel_ms": kernel_ms}
        finally:
            self.bp.refg_bp_destroy(h)

    def filter(self, views_t, table_t, H_t, W):
        """cuFFT plugin on torch CUDA tensors (views modified in place by the cos weight)."""
        import torch

        n, h, w = views_t.shape
        dst = torch.empty_like(views_t)
        r = self.flt.refg_filter(views_t.data_ptr(), dst.data_ptr(), table_t.data_ptr(),
                                 H_t.data_ptr(), w, h, n, W)
        assert r == 0, r
        return dst
