"""fdk_b200 -- B200-native FDK cone-beam reconstruction behind the reference's plugin API.

Host-side mirror of the reference interfaces (peng-ac/fdk):
  Parameter                  common/type.h Parameter (geometry, filter, cos table, matrices)
  FilterEngine               Filterlib/FilterLib.h FilterEngine
  filter_row_real32 / correct_image_real32
                             FilterlibCufft/cudaFftFilter.cuh
  BackProjectionFDK          cudaBP/backprojection.cuh BackProjectionFDK
  reconstruct_conebeam       cudaBP/rtkCudaFDKBackProjectionImageFilter.cu CUDA_reconstruct_conebeam
  Reconstructor              single-GPU streaming FDK (cuFDK filter -> BP handoff)
All compute runs in libfdk_b200.so (CUDA, sm_100a); there is no CPU fallback.
"""
from ._lib import (BP_FP32, BP_FP32_EXACT, BP_MIXED, DTYPE_F16, DTYPE_F32, LAYOUT_MIRROR, LAYOUT_ROWS,
                   LAYOUT_TRANSPOSED, FdkError, device_count, lib)
from .backprojection import BackProjectionFDK, BoxT, reconstruct_conebeam
from .filter import FilterEngine, ToeplitzFilter, correct_image_real32, filter_row_real32, toeplitz_matrix
from .geometry import Parameter, config, default_parameter
from .recon import Reconstructor

__all__ = [
    "Parameter", "config", "default_parameter", "FilterEngine", "ToeplitzFilter", "toeplitz_matrix",
    "correct_image_real32", "filter_row_real32",
    "BackProjectionFDK", "BoxT", "reconstruct_conebeam", "Reconstructor", "FdkError", "device_count", "lib",
    "BP_FP32_EXACT", "BP_FP32", "BP_MIXED", "DTYPE_F32", "DTYPE_F16", "LAYOUT_ROWS", "LAYOUT_TRANSPOSED",
    "LAYOUT_MIRROR",
]
