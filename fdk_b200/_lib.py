"""ctypes binding of libfdk_b200.so (the C ABI declared in include/fdk.h).

The library is built in-tree (``python -m fdk_b200.build``).  There is no fallback: if the
shared object is missing or does not load, importing this module raises, so no CPU or
library path can silently stand in for the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdk_b200.so")

FDK_OK = 0
ERRORS = {
    -1: "FDK_ERR_INVALID_ARG",
    -2: "FDK_ERR_CUDA",
    -3: "FDK_ERR_OUT_OF_MEMORY",
    -4: "FDK_ERR_TIMEOUT",
    -5: "FDK_ERR_UNSUPPORTED",
    -6: "FDK_ERR_NO_DEVICE",
    -7: "FDK_ERR_DEVICE_CHECK",
    -8: "FDK_ERR_IO",
}

# filter windows (s_FILTER_TYPE order, common/type.h:4619-4626)
FILTERS = {"none": 0, "ram-lak": 1, "shepp-logan": 2, "cosine": 3, "hamming": 4, "hann": 5}
DTYPE_F32, DTYPE_F16 = 0, 1
LAYOUT_ROWS, LAYOUT_TRANSPOSED, LAYOUT_MIRROR = 0, 1, 2
BP_FP32_EXACT, BP_FP32, BP_MIXED = 0, 1, 2
PRECISIONS = {"fp32_exact": BP_FP32_EXACT, "fp32": BP_FP32, "mixed": BP_MIXED}

# every symbol include/fdk.h declares (tests check the library exports all of them)
EXPORTED = [
    "fdk_last_error", "fdk_abi_version", "fdk_device_count",
    "fdk_geometry_default", "fdk_filter_length", "fdk_filter_design", "fdk_angular_ramp_factor",
    "fdk_cos_table", "fdk_csc_table", "fdk_view_angles", "fdk_projection_matrices",
    "fdk_filter_create", "fdk_filter_filtering", "fdk_filter_run_device", "fdk_filter_destroy",
    "fdk_correct_image_real32", "fdk_filter_row_real32", "fdk_filter_row_real32_noalloc",
    "fdk_bp_create", "fdk_bp_bp", "fdk_bp_bp_device", "fdk_bp_get_volume", "fdk_bp_volume_device",
    "fdk_bp_sample", "fdk_bp_stats", "fdk_bp_reset", "fdk_bp_destroy",
    "fdk_rtk_reconstruct_conebeam", "fdk_rtk_backproject_device", "fdk_rtk_sync",
    "fdk_recon_create", "fdk_recon_create_slab", "fdk_recon_stream", "fdk_recon_push", "fdk_recon_push_device",
    "fdk_recon_push_views", "fdk_recon_push_device_views",
    "fdk_recon_push_folder", "fdk_recon_flush", "fdk_recon_filter_kind", "fdk_recon_bp_kernel", "fdk_recon_sync",
    "fdk_recon_get_volume", "fdk_recon_sample", "fdk_recon_stats", "fdk_recon_launch_count", "fdk_recon_reset", "fdk_recon_destroy",
    "fdk_phantom_project", "fdk_forward_project", "fdk_probe_smem", "fdk_probe_fma",
    "fdk_nn_param_count", "fdk_nn_forward", "fdk_nn_backward", "fdk_adam_step", "fdk_transmission_noise",
    "fdk_voxelize", "fdk_rows_to_mirror", "fdk_volume_mse", "fdk_bp_adjoint",
    "fdk_proj_path", "fdk_load_proj_folder", "fdk_save_proj_folder", "fdk_save_volume", "fdk_load_volume",
    "fdk_save_volume_slices",
    "fdk_toeplitz_create", "fdk_toeplitz_run_device", "fdk_toeplitz_check", "fdk_toeplitz_matrix",
    "fdk_toeplitz_destroy",
]


class FdkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Geometry(C.Structure):
    """fdk_geometry -- the reference's Parameter (common/type.h:4627-4895) as a plain struct."""

    _fields_ = [
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("nu", C.c_int64), ("nv", C.c_int64),
        ("du", C.c_double), ("dv", C.c_double),
        ("offset_nu", C.c_double), ("offset_nv", C.c_double),
        ("sid", C.c_double), ("sod", C.c_double),
        ("direction", C.c_int64), ("scan_angle", C.c_double), ("n_proj", C.c_int64),
        ("volume_position_angle", C.c_double),
        ("filter_type", C.c_int32), ("reserved", C.c_int32),
    ]


class Box(C.Structure):
    """fdk_box -- geo::BoxT<size_t> (cudaBP/backprojection.cuh:66-116)."""

    _fields_ = [(n, C.c_uint64) for n in ("x", "y", "z", "width", "height", "depth")]


class DataRef(C.Structure):
    """fdk_dataref -- DataRef<float> (FilterlibCufft/cudaBackProjection.cuh:121-230)."""

    _fields_ = [("data", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32),
                ("depth", C.c_int32), ("pitch", C.c_int32)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fdk_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, f64p = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_double)
    G = C.POINTER(Geometry)
    sig = {
        "fdk_last_error": ([], C.c_char_p),
        "fdk_abi_version": ([], C.c_int),
        "fdk_device_count": ([C.POINTER(C.c_int)], C.c_int),
        "fdk_geometry_default": ([G], None),
        "fdk_filter_length": ([i64], i64),
        "fdk_filter_design": ([i32, i64, i32, vp, i64], C.c_int),
        "fdk_angular_ramp_factor": ([G, f64p], C.c_int),
        "fdk_cos_table": ([G, vp], C.c_int),
        "fdk_csc_table": ([G, vp], C.c_int),
        "fdk_view_angles": ([G, vp], C.c_int),
        "fdk_projection_matrices": ([G, vp, vp], C.c_int),
        "fdk_filter_create": ([C.POINTER(vp), vp, vp, i64, i64, i64, i32, i32], C.c_int),
        "fdk_filter_filtering": ([vp, vp, vp, i32], C.c_int),
        "fdk_filter_run_device": ([vp, vp, vp, i64, i32, i32, C.c_float, vp], C.c_int),
        "fdk_filter_destroy": ([vp], C.c_int),
        "fdk_correct_image_real32": ([C.POINTER(DataRef)] * 3, C.c_int),
        "fdk_filter_row_real32": ([C.POINTER(DataRef)] * 3, C.c_int),
        "fdk_filter_row_real32_noalloc": ([C.POINTER(DataRef)] * 3, C.c_int),
        "fdk_bp_create": ([C.POINTER(vp), i32, i32, i32, i32, i32, i32, C.POINTER(Box), C.POINTER(Box),
                           i32, i32], C.c_int),
        "fdk_bp_bp": ([vp, i32, vp, i32, i32, vp, i32], C.c_int),
        "fdk_bp_bp_device": ([vp, vp, i32, vp, i32, vp], C.c_int),
        "fdk_bp_get_volume": ([vp, vp, i64], C.c_int),
        "fdk_bp_volume_device": ([vp, C.POINTER(vp), C.POINTER(i64)], C.c_int),
        "fdk_bp_sample": ([vp, vp, i64, vp], C.c_int),
        "fdk_bp_stats": ([vp, C.POINTER(i64), f64p], C.c_int),
        "fdk_bp_reset": ([vp], C.c_int),
        "fdk_bp_destroy": ([vp], C.c_int),
        "fdk_rtk_reconstruct_conebeam": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "fdk_rtk_backproject_device": ([vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "fdk_rtk_sync": ([vp], C.c_int),
        "fdk_recon_create": ([C.POINTER(vp), G, i32, i32, i32], C.c_int),
        "fdk_recon_create_slab": ([C.POINTER(vp), G, i64, i64, i32, i32, i32], C.c_int),
        "fdk_recon_stream": ([vp, C.POINTER(vp)], C.c_int),
        "fdk_recon_push": ([vp, vp, i64, i64], C.c_int),
        "fdk_recon_push_device": ([vp, vp, i64, i64], C.c_int),
        "fdk_recon_push_views": ([vp, vp, vp, i64], C.c_int),
        "fdk_recon_push_device_views": ([vp, vp, vp, i64], C.c_int),
        "fdk_recon_push_folder": ([vp, C.c_char_p, i64, i64, i32, i32, i32], C.c_int),
        "fdk_recon_flush": ([vp], C.c_int),
        "fdk_recon_filter_kind": ([vp, C.POINTER(i32)], C.c_int),
        "fdk_recon_bp_kernel": ([vp, C.POINTER(i32)], C.c_int),
        "fdk_recon_sync": ([vp, i64], C.c_int),
        "fdk_recon_get_volume": ([vp, vp, i64], C.c_int),
        "fdk_recon_sample": ([vp, vp, i64, vp], C.c_int),
        "fdk_recon_stats": ([vp, f64p, f64p, C.POINTER(i64)], C.c_int),
        "fdk_recon_launch_count": ([vp, C.POINTER(i64)], C.c_int),
        "fdk_recon_reset": ([vp], C.c_int),
        "fdk_recon_destroy": ([vp], C.c_int),
        "fdk_phantom_project": ([G, vp, i32, i64, i64, vp, vp], C.c_int),
        "fdk_forward_project": ([G, vp, i64, i64, vp, vp], C.c_int),
        "fdk_nn_param_count": ([], C.c_int),
        "fdk_nn_forward": ([vp, vp, vp, i64, i32, C.c_float, vp], C.c_int),
        "fdk_nn_backward": ([vp, vp, vp, vp, i64, i32, C.c_float, vp], C.c_int),
        "fdk_adam_step": ([vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, i64, vp], C.c_int),
        "fdk_transmission_noise": ([vp, i64, C.c_double, C.c_double, C.c_uint64, vp], C.c_int),
        "fdk_voxelize": ([G, vp, i32, vp, vp], C.c_int),
        "fdk_rows_to_mirror": ([vp, vp, i64, i32, i32, vp], C.c_int),
        "fdk_volume_mse": ([vp, vp, vp, i32, i32, i32, f64p, vp], C.c_int),
        "fdk_bp_adjoint": ([G, vp, vp, i32, vp, vp], C.c_int),
        "fdk_proj_path": ([C.c_char_p, i64, i32, i32, C.c_char_p, i32], C.c_int),
        "fdk_load_proj_folder": ([C.c_char_p, i32, i32, i64, i64, i32, i32, vp, i32], C.c_int),
        "fdk_save_proj_folder": ([C.c_char_p, vp, i32, i32, i64, i64, i32, i32], C.c_int),
        "fdk_save_volume": ([C.c_char_p, vp, i32, i32, i32], C.c_int),
        "fdk_load_volume": ([C.c_char_p, vp, i64, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)], C.c_int),
        "fdk_save_volume_slices": ([C.c_char_p, vp, i32, i32, i32, i32, i32], C.c_int),
        "fdk_toeplitz_create": ([C.POINTER(vp), vp, vp, i64, i64, i64, i32, i32, i32, C.c_float, i32], C.c_int),
        "fdk_toeplitz_run_device": ([vp, vp, vp, i64, i32, C.c_float, vp], C.c_int),
        "fdk_toeplitz_check": ([vp], C.c_int),
        "fdk_toeplitz_matrix": ([vp, i64, i64, i32, vp], C.c_int),
        "fdk_toeplitz_destroy": ([vp], C.c_int),
        "fdk_probe_smem": ([i32, f64p], C.c_int),
        "fdk_probe_fma": ([i32, f64p], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != FDK_OK:
        msg = lib().fdk_last_error()
        raise FdkError(rc, msg.decode() if msg else "")


def probe_peaks(device: int = 0) -> dict:
    """Measured shared-memory bandwidth (GB/s) and FP32 FMA rate (TFLOP/s) of the device."""
    a, b = C.c_double(), C.c_double()
    check(lib().fdk_probe_smem(device, C.byref(a)))
    check(lib().fdk_probe_fma(device, C.byref(b)))
    return {"smem_gbs": a.value, "fp32_tflops": b.value}


def device_count() -> int:
    n = C.c_int(0)
    check(lib().fdk_device_count(C.byref(n)))
    return n.value
