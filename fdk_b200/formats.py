"""On-disk formats of the reconstruction path (host code in libfdk_b200.so, no GPU needed).

  proj_path / load_proj_folder / save_proj_folder
      one raw FP32 file per view, nv x nu, u fastest, "img%04d.raw" with file index
      view * step + start (Parameter::GetProjPath, common/type.h:4847-4851;
      LoadProjectionImageFolder 1797-1828; SaveToFolder 3848-3861)
  save_volume / load_volume
      ".vol": int32 nx, ny, nz then the FP32 voxels [z][y][x] (VolumeT::Save/Load, 3256-3313)
  save_volume_slices
      one raw FP32 file of ny x nx per slice, "%06d.raw" by global slice index (the slice writer
      of cuFDK/mpiFDK.cpp:548-576)

Folders are given with or without a trailing '/'; file names are appended to them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .recon import _folder_arg


def proj_path(folder: str, view: int, step: int = 1, start: int = 0) -> str:
    buf = C.create_string_buffer(4096)
    check(lib().fdk_proj_path(_folder_arg(folder), view, step, start, buf, len(buf)))
    return buf.value.decode()


def load_proj_folder(folder: str, nu: int, nv: int, count: int, first: int = 0, step: int = 1, start: int = 0,
                     out: np.ndarray | None = None, threads: int = 0) -> np.ndarray:
    """Views first..first+count-1 as (count, nv, nu) float32 (into `out`, e.g. pinned, if given)."""
    if out is None:
        out = np.empty((count, nv, nu), np.float32)
    if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < count * nu * nv:
        raise ValueError("out must be C-contiguous float32 with room for count views")
    check(lib().fdk_load_proj_folder(_folder_arg(folder), nu, nv, first, count, step, start, out.ctypes.data,
                                     threads))
    return out


def save_proj_folder(folder: str, views: np.ndarray, first: int = 0, step: int = 1, threads: int = 0) -> None:
    v = np.ascontiguousarray(views, np.float32)
    n, nv, nu = v.shape
    check(lib().fdk_save_proj_folder(_folder_arg(folder), v.ctypes.data, nu, nv, first, n, step, threads))


def save_volume(path: str, vol: np.ndarray) -> None:
    v = np.ascontiguousarray(vol, np.float32)
    nz, ny, nx = v.shape
    check(lib().fdk_save_volume(path.encode(), v.ctypes.data, nx, ny, nz))


def load_volume(path: str) -> np.ndarray:
    nx, ny, nz = C.c_int32(), C.c_int32(), C.c_int32()
    check(lib().fdk_load_volume(path.encode(), None, 0, C.byref(nx), C.byref(ny), C.byref(nz)))
    out = np.empty((nz.value, ny.value, nx.value), np.float32)
    check(lib().fdk_load_volume(path.encode(), out.ctypes.data, out.size, C.byref(nx), C.byref(ny), C.byref(nz)))
    return out


def save_volume_slices(folder: str, vol: np.ndarray, z0: int = 0, threads: int = 0) -> None:
    v = np.ascontiguousarray(vol, np.float32)
    depth, ny, nx = v.shape
    check(lib().fdk_save_volume_slices(_folder_arg(folder), v.ctypes.data, nx, ny, z0, depth, threads))
