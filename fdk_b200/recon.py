"""Reconstructor: end-to-end streaming FDK on one GPU (cosine weight, ramp filter,
backprojection), the single-GPU form of cuFDK's filter -> BP handoff (cuFDK/mpiFDK.cpp:58-317).

The whole volume is reconstructed as one mirror-symmetric slab pair; with ``slab=(top_z,
depth)`` only that pair (one rank of DivVolume, see ``fdk_b200.shard``)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PRECISIONS, check, lib


class Reconstructor:
    def __init__(self, param, precision: str = "mixed", batch: int = 128, device: int = 0, slab=None):
        self.param = param
        self.precision = precision
        self._g = param.to_c()
        self._h = C.c_void_p()
        if slab is None:
            slab = (0, param.nz // 2)
        self.slab = (int(slab[0]), int(slab[1]))
        check(lib().fdk_recon_create_slab(C.byref(self._h), C.byref(self._g), self.slab[0], self.slab[1],
                                          PRECISIONS[precision], batch, device))

    @property
    def depth(self) -> int:
        """Storage depth of the slab pair (top + bottom)."""
        return 2 * self.slab[1]

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().fdk_recon_stream(self._h, C.byref(s)))
        return s.value or 0

    def push(self, views: np.ndarray, first: int) -> None:
        """Raw views (n, nv, nu) float32 in host memory (pinned memory overlaps best)."""
        if views.dtype != np.float32 or not views.flags.c_contiguous:
            raise ValueError("views must be C-contiguous float32")
        check(lib().fdk_recon_push(self._h, views.ctypes.data, first, views.shape[0]))

    def push_ptr(self, host_ptr: int, first: int, n: int) -> None:
        check(lib().fdk_recon_push(self._h, host_ptr, first, n))

    def push_views(self, views: np.ndarray, ids) -> None:
        """Raw views (n, nv, nu) float32 in host memory with view indices ids (any order)."""
        if views.dtype != np.float32 or not views.flags.c_contiguous:
            raise ValueError("views must be C-contiguous float32")
        self.push_views_ptr(views.ctypes.data, ids)

    def push_views_ptr(self, host_ptr: int, ids) -> None:
        ids = np.ascontiguousarray(ids, np.int64)
        check(lib().fdk_recon_push_views(self._h, host_ptr, ids.ctypes.data, len(ids)))

    def push_device_views(self, dev_ptr: int, ids) -> None:
        """Raw views in device memory, one after another, with view indices ids (any order)."""
        ids = np.ascontiguousarray(ids, np.int64)
        check(lib().fdk_recon_push_device_views(self._h, dev_ptr, ids.ctypes.data, len(ids)))

    @property
    def filter_kind(self) -> str:
        """'fft' or 'tensor' (the split-FP16 tcgen05 GEMM filter)."""
        k = C.c_int32()
        check(lib().fdk_recon_filter_kind(self._h, C.byref(k)))
        return "tensor" if k.value == 1 else "fft"

    @property
    def bp_kernel(self) -> str:
        """'exact', 'staged' or 'quarter-turn' (the staged kernel plus the quarter-turn kernel for
        views whose three quarter-turn partners share their batch)."""
        k = C.c_int32()
        check(lib().fdk_recon_bp_kernel(self._h, C.byref(k)))
        return ("exact", "staged", "quarter-turn")[k.value]

    def flush(self) -> None:
        """Backproject every filtered view still waiting (a held full batch and the filling one)
        now (asynchronous)."""
        check(lib().fdk_recon_flush(self._h))

    def push_folder(self, folder: str, first: int, n: int, step: int = 1, start: int = 0, threads: int = 0) -> None:
        """Views first..first+n-1 from a projection folder (img%04d.raw, view v in file v*step+start),
        read into pinned staging while the previous batch is copied and reconstructed."""
        check(lib().fdk_recon_push_folder(self._h, _folder_arg(folder), first, n, step, start, threads))

    def push_device(self, dev_ptr: int, first: int, n: int) -> None:
        check(lib().fdk_recon_push_device(self._h, dev_ptr, first, n))

    def sync(self, timeout_ms: int = 0) -> None:
        check(lib().fdk_recon_sync(self._h, timeout_ms))

    def volume(self, out: np.ndarray | None = None) -> np.ndarray:
        """[zs][y][x]: the full volume [z][y][x] for the default slab pair."""
        p = self.param
        n = p.nx * p.ny * self.depth
        if out is None:
            out = np.empty(n, np.float32)
        check(lib().fdk_recon_get_volume(self._h, out.ctypes.data, n))
        return out.reshape(self.depth, p.ny, p.nx)

    def volume_into(self, host_ptr: int) -> None:
        p = self.param
        check(lib().fdk_recon_get_volume(self._h, host_ptr, p.nx * p.ny * self.depth))

    def sample(self, xyz: np.ndarray) -> np.ndarray:
        """Values at voxels xyz ((n, 3) int (x, y, z) of the whole volume) after a sync; voxels
        outside the slab pair read NaN.  Reads n values instead of the whole volume."""
        xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
        out = np.empty(len(xyz), np.float32)
        check(lib().fdk_recon_sample(self._h, xyz.ctypes.data, len(xyz), out.ctypes.data))
        return out

    def stats(self):
        bp, fl, n = C.c_double(), C.c_double(), C.c_int64()
        check(lib().fdk_recon_stats(self._h, C.byref(bp), C.byref(fl), C.byref(n)))
        return {"bp_ms": bp.value, "filter_ms": fl.value, "views": n.value}

    @property
    def launch_count(self) -> int:
        """Kernel launches (filter and backprojection) since creation or the last reset."""
        n = C.c_int64()
        check(lib().fdk_recon_launch_count(self._h, C.byref(n)))
        return n.value

    def reset(self) -> None:
        check(lib().fdk_recon_reset(self._h))

    def close(self):
        if self._h:
            lib().fdk_recon_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _folder_arg(folder: str) -> bytes:
    """The C entry points append file names to the folder string, as the reference does."""
    return (folder if folder.endswith("/") else folder + "/").encode()
