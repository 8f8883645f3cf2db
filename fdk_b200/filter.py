"""Filter plugins over the C ABI.

* ``FilterEngine`` mirrors Filterlib/FilterLib.h:148-203 (the production IPP plugin):
  ``FilterEngine(cos_image_table, fft_kernel_real_f32).Filtering(src, dst, transpose)``.
* ``filter_row_real32`` / ``correct_image_real32`` mirror the cuFFT plugin
  (FilterlibCufft/cudaFftFilter.cuh:6-8) on device buffers.
* ``ToeplitzFilter`` is the same filter as a tensor-core GEMM (no reference counterpart).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (DTYPE_F16, DTYPE_F32, LAYOUT_MIRROR, LAYOUT_ROWS, LAYOUT_TRANSPOSED, DataRef, check,
                   lib)


class FilterEngine:
    """Cosine weight + ramp filter + optional transpose of one view (Filterlib/FilterLib.h).

    ``pad_edge`` is the number of edge samples averaged into the constant pad: 4 as the IPP
    plugin (FilterLib.h:38,44), 3 as the cuFFT plugin (cudaFftFilter.cu:25,29).
    """

    def __init__(self, cos_image_table, fft_kernel_real_f32, pad_edge: int = 4, device: int = 0):
        cos = None if cos_image_table is None else np.ascontiguousarray(cos_image_table, np.float32)
        H = np.ascontiguousarray(fft_kernel_real_f32, np.float32)
        if cos is None:
            raise ValueError("cos_image_table is required (pass ones to disable weighting)")
        self.nv, self.nu = cos.shape
        self.W = len(H)
        self._h = C.c_void_p()
        check(lib().fdk_filter_create(C.byref(self._h), cos.ctypes.data, H.ctypes.data, self.nu, self.nv, self.W,
                                      pad_edge, device))

    def Filtering(self, src: np.ndarray, dst: np.ndarray, transpose: bool = False) -> "FilterEngine":
        """src (nv, nu) float32 is cosine-weighted in place, as in the reference (FilterLib.h:181)."""
        if src.dtype != np.float32 or not src.flags.c_contiguous or src.shape != (self.nv, self.nu):
            raise ValueError("src must be a C-contiguous float32 (nv, nu) array")
        want = (self.nu, self.nv) if transpose else (self.nv, self.nu)
        if dst.dtype != np.float32 or not dst.flags.c_contiguous or dst.shape != want:
            raise ValueError(f"dst must be a C-contiguous float32 {want} array")
        check(lib().fdk_filter_filtering(self._h, src.ctypes.data, dst.ctypes.data, int(bool(transpose))))
        return self

    def run_device(self, src_ptr: int, dst_ptr: int, n_views: int, layout: int = LAYOUT_TRANSPOSED,
                   dtype: int = DTYPE_F32, out_scale: float = 1.0, stream: int = 0) -> None:
        """Batch filter on device buffers (cosine weight applied on the fly); every output
        sample is multiplied by out_scale (keep FP16 outputs in range)."""
        check(lib().fdk_filter_run_device(self._h, src_ptr, dst_ptr, n_views, layout, dtype, out_scale, stream))

    def close(self):
        if self._h:
            lib().fdk_filter_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ref(ptr: int, width: int, height: int, depth: int, pitch: int | None = None) -> DataRef:
    return DataRef(ptr, width, height, depth, width if pitch is None else pitch)


def correct_image_real32(src, table, dst) -> None:
    """CorrectImage_Real32 on torch CUDA tensors: dst = src * table (per view)."""
    d, h, w = src.shape
    check(lib().fdk_correct_image_real32(C.byref(_ref(src.data_ptr(), w, h, d)),
                                         C.byref(_ref(table.data_ptr(), w, h, 1)),
                                         C.byref(_ref(dst.data_ptr(), w, h, dst.shape[0]))))


def filter_row_real32(src, dst, filt) -> None:
    """FilterRow_Real32 on torch CUDA tensors: ramp-filter every row (pad = mean of 3 edge samples)."""
    d, h, w = src.shape
    check(lib().fdk_filter_row_real32(C.byref(_ref(src.data_ptr(), w, h, d)),
                                      C.byref(_ref(dst.data_ptr(), w, h, dst.shape[0])),
                                      C.byref(_ref(filt.data_ptr(), filt.numel(), 1, 1))))


__all__ = ["FilterEngine", "correct_image_real32", "filter_row_real32", "LAYOUT_ROWS", "LAYOUT_TRANSPOSED",
           "LAYOUT_MIRROR", "DTYPE_F32", "DTYPE_F16"]


class ToeplitzFilter:
    """The row filter as a GEMM on the tensor cores (fdk_toeplitz_*): y = M (in_scale * cos * p)
    per row, M the nu x nu matrix of the fused filter, FP16 or BF16 operands, FP32 accumulation,
    FP16 output (ROWS or MIRROR layout).  No reference counterpart."""

    def __init__(self, cos_table: np.ndarray, H: np.ndarray, pad_edge: int = 4, dtype: str = "f16",
                 in_scale: float = 1.0, device: int = 0, split: bool = False):
        cos = np.ascontiguousarray(cos_table, np.float32)
        self.nv, self.nu = cos.shape
        h = np.ascontiguousarray(H, np.float64)
        self._h = C.c_void_p()
        check(lib().fdk_toeplitz_create(C.byref(self._h), cos.ctypes.data, h.ctypes.data, self.nu, self.nv, h.size,
                                        pad_edge, 1 if dtype == "bf16" else 0, 1 if split else 0, in_scale, device))

    def run_device(self, src_ptr: int, dst_ptr: int, n_views: int, layout: int = LAYOUT_ROWS, out_scale: float = 1.0,
                   stream: int = 0) -> None:
        check(lib().fdk_toeplitz_run_device(self._h, src_ptr, dst_ptr, n_views, layout, out_scale, stream))

    def check(self) -> None:
        check(lib().fdk_toeplitz_check(self._h))

    def close(self) -> None:
        if self._h:
            lib().fdk_toeplitz_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def toeplitz_matrix(H: np.ndarray, nu: int, pad_edge: int = 4) -> np.ndarray:
    """FP64 filter matrix M (nu x nu) of the fused filter with response H (W taps)."""
    h = np.ascontiguousarray(H, np.float64)
    out = np.empty((nu, nu), np.float64)
    check(lib().fdk_toeplitz_matrix(h.ctypes.data, h.size, nu, pad_edge, out.ctypes.data))
    return out
