"""Timing of the RTK drop-in on device-resident views (`fdk_rtk_backproject_device`): a 512^3
FP32 volume from 32 views of 512^2 (the c2 geometry at that size, a seeded 20-ellipsoid phantom
projected on the GPU), circular matrices and tilted ones (m[2] += 0.02 std(m[0]), m[10] += 1e-3,
so u and w depend on z).  One JSON line per geometry and kernel: the staged kernel ("tma") and
the L1-gather kernel ("l1", FDK_RTK_KERNEL=l1); 3 warm-up and 10 timed launches, CUDA events.

  python -m fdk_b200.rtk_bench [tma] [l1]
"""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import numpy as np  # noqa: E402
import torch  # noqa: E402

import fdk_b200 as F  # noqa: E402
from fdk_b200.backprojection import rtk_backproject_device, rtk_sync  # noqa: E402
from fdk_b200.phantom import phantom_for, project  # noqa: E402


def main():
    n, W, views = 512, 512, 32
    p = F.config("c2")
    p.nx = p.ny = p.nz = n
    p.nu = p.nv = W
    p.nProj = views
    dev = torch.empty((views, W, W), dtype=torch.float32, device="cuda")
    project(p, phantom_for(p, 2, 20), 0, views, dev.data_ptr())
    vin = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    vout = torch.empty_like(vin)
    size = (W, W, views), (n, n, n)
    for geo in ("circular", "tilted"):
        mats = p.proj_matrices(np.float64)
        if geo == "tilted":
            mats[:, 2] += 0.02 * mats[:, 0].std()
            mats[:, 10] += 1e-3
        mats = mats.astype(np.float32)
        for kern in sys.argv[1:] or ["tma", "l1"]:
            if kern == "l1":
                os.environ["FDK_RTK_KERNEL"] = "l1"
            else:
                os.environ.pop("FDK_RTK_KERNEL", None)
            for _ in range(3):
                rtk_backproject_device(*size, mats, vin.data_ptr(), vout.data_ptr(), dev.data_ptr())
            rtk_sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                rtk_backproject_device(*size, mats, vin.data_ptr(), vout.data_ptr(), dev.data_ptr())
            e1.record()
            e1.synchronize()
            rtk_sync()
            ms = e0.elapsed_time(e1) / 10
            print(json.dumps({"geometry": geo, "kernel": kern, "ms": ms, "gups": n ** 3 * views / (ms * 1e-3) / 1e9}),
                  flush=True)


if __name__ == "__main__":
    main()
