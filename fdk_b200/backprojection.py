"""Backprojection plugins over the C ABI.

* ``BackProjectionFDK`` mirrors cudaBP/backprojection.cuh:246-271
  (ctor(projW, projH, projCount, nx, ny, nz, subTop, subBottom), BP, GetVolumeData,
  nBpCount, fKernelTime).
* ``reconstruct_conebeam`` mirrors BackProjectionRTK::CUDA_reconstruct_conebeam
  (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:200-206).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import LAYOUT_MIRROR, LAYOUT_TRANSPOSED, PRECISIONS, Box, check, lib


def BoxT(x, y, z, width, height, depth) -> Box:
    """geo::BoxT<size_t>(x, y, z, width, height, depth)."""
    return Box(x, y, z, width, height, depth)


class BackProjectionFDK:
    MAX_PROJ = 32

    def __init__(self, projWidth: int, projHeight: int, projCount: int, nx: int, ny: int, nz: int,
                 subTop: Box, subBottom: Box, precision: str = "fp32_exact", device: int = 0):
        self.subTop, self.subBottom = subTop, subBottom
        self.precision = precision
        self._h = C.c_void_p()
        check(lib().fdk_bp_create(C.byref(self._h), projWidth, projHeight, projCount, nx, ny, nz, C.byref(subTop),
                                  C.byref(subBottom), PRECISIONS[precision], device))

    @property
    def volume_size(self) -> int:
        return int(self.subTop.width * self.subTop.height * (self.subTop.depth + self.subBottom.depth))

    def BP(self, TRANSPOSE: int, pProjData: np.ndarray, width: int, height: int, pProjMat: np.ndarray,
           nProj: int) -> bool:
        p = np.ascontiguousarray(pProjData, np.float32)
        m = np.ascontiguousarray(pProjMat, np.float32)
        if p.size < width * height * nProj or m.size < 12 * nProj:
            raise ValueError("projection or matrix buffer too small")
        check(lib().fdk_bp_bp(self._h, TRANSPOSE, p.ctypes.data, width, height, m.ctypes.data, nProj))
        return True

    def BP_device(self, dev_ptr: int, layout: int, pProjMat: np.ndarray, nProj: int, stream: int = 0) -> None:
        m = np.ascontiguousarray(pProjMat, np.float32)
        check(lib().fdk_bp_bp_device(self._h, dev_ptr, layout, m.ctypes.data, nProj, stream))

    def GetVolumeData(self, pVol: np.ndarray | None = None, size: int | None = None) -> np.ndarray:
        """Sub-volume as [zs][y][x] (zs = top slab then bottom slab, ascending)."""
        n = self.volume_size
        out = np.empty(n, np.float32) if pVol is None else pVol
        check(lib().fdk_bp_get_volume(self._h, out.ctypes.data, n if size is None else size))
        D = int(self.subTop.depth + self.subBottom.depth)
        return out.reshape(D, int(self.subTop.height), int(self.subTop.width))

    def volume_device(self):
        p, n = C.c_void_p(), C.c_int64()
        check(lib().fdk_bp_volume_device(self._h, C.byref(p), C.byref(n)))
        return p.value, n.value

    def stats(self):
        n, ms = C.c_int64(), C.c_double()
        check(lib().fdk_bp_stats(self._h, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    @property
    def nBpCount(self) -> int:
        return self.stats()[0]

    @property
    def fKernelTime(self) -> float:
        return self.stats()[1]

    def reset(self):
        check(lib().fdk_bp_reset(self._h))

    def close(self):
        if self._h:
            lib().fdk_bp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reconstruct_conebeam(proj_size, vol_size, matrices: np.ndarray, dev_vol_in: int, dev_vol_out: int,
                         proj: np.ndarray) -> None:
    """CUDA_reconstruct_conebeam: dev_vol_out = dev_vol_in + BP(proj) (host proj, device volumes)."""
    ps = (C.c_int32 * 3)(*proj_size)
    vs = (C.c_int32 * 3)(*vol_size)
    m = np.ascontiguousarray(matrices, np.float32)
    p = np.ascontiguousarray(proj, np.float32)
    check(lib().fdk_rtk_reconstruct_conebeam(ps, vs, m.ctypes.data, dev_vol_in, dev_vol_out, p.ctypes.data))


def rtk_backproject_device(proj_size, vol_size, matrices: np.ndarray, dev_vol_in: int, dev_vol_out: int,
                           dev_proj: int, stream: int = 0) -> None:
    """The same as reconstruct_conebeam on device-resident views (up to 128), asynchronous."""
    ps = (C.c_int32 * 3)(*proj_size)
    vs = (C.c_int32 * 3)(*vol_size)
    m = np.ascontiguousarray(matrices, np.float32)
    check(lib().fdk_rtk_backproject_device(ps, vs, m.ctypes.data, dev_vol_in, dev_vol_out, dev_proj, stream))


def rtk_sync(stream: int = 0) -> None:
    """Wait for stream; raise if the staged RTK kernel reported a device-side failure."""
    check(lib().fdk_rtk_sync(stream))


__all__ = ["BackProjectionFDK", "BoxT", "reconstruct_conebeam", "rtk_backproject_device", "rtk_sync",
           "LAYOUT_MIRROR", "LAYOUT_TRANSPOSED"]
