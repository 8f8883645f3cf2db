"""Writes tests/golden/ref_gpu.npz: outputs of the reference's own cuFFT filter plugin compiled for
sm_100a by oracle/build_ref.sh (oracle/_ref/libref_gpu_filter.so), on small seeded inputs.  Needs
a CUDA GPU.

    python tests/golden/make_golden_gpu.py

The plugin's CorrectImage_Real32 then FilterRow_Real32 (FilterlibCufft/cudaFftFilter.cu:270-384)
ran on 3 seeded views of 64 x 16; the cosine table and the response it was given are stored
beside its output.  tests/test_golden.py checks the oracle's FP64 row filter against them on the
CPU, to 5e-6.

The reference's backprojection (cudaFdkBP through BackProjectionFDK) is checked live on the GPU
instead (tests/test_gpu_bp.py: our exact kernel and the oracle's emulation against it, bit for
bit), at sizes its code accepts: its lanes run along the top slab's depth, and a lane past the
depth returns (cudaBP/backprojectionFDK.cu:64-66) before the warp shuffle that hands each view's
(U, 1/w) from lane s to the others (:80-98), so at depths that are not a multiple of 32 the views
whose lanes have returned read undefined values (a 32^3 volume, depth 16, came out different from
the oracle at 86% of its voxels); and GetVolumeData's TransformVolume (:139-149) asserts a slab
height that is a multiple of 32 and a depth and width that are multiples of 4 (a 16 x 16 x 64
volume stopped there).  Our kernels take any of these sizes."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

FLT_NU, FLT_NV, FLT_VIEWS, FLT_SEED = 64, 16, 3, 7


def filter_views():
    rng = np.random.default_rng(FLT_SEED)
    return (rng.standard_normal((FLT_VIEWS, FLT_NV, FLT_NU)) * 10).astype(np.float32)


def main() -> None:
    import torch

    from tests.helpers import small_param

    assert torch.cuda.is_available(), "needs a CUDA GPU"
    R = O.RefGPU()
    q = small_param(64, FLT_NU, FLT_NV, 3)
    out = {"flt_cos": q.cos_sigma, "flt_H": q.fft_kernel_real_f32}
    views = torch.from_numpy(filter_views()).cuda()
    out["flt_out"] = R.filter(views, torch.from_numpy(q.cos_sigma).cuda(), torch.from_numpy(q.fft_kernel_real_f32).cuda(),
                              len(q.fft_kernel_real_f32)).cpu().numpy()
    path = os.path.join(os.environ.get("GOLDEN_OUT", HERE), "ref_gpu.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
