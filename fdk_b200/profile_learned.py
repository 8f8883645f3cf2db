"""Profiling driver for the learned-filter training step on the C5 geometry (256^3 volume, 90
views of 256^2): one noisy scan, then `n_steps` forward + loss + gradient passes (network
forward, backprojection, volume MSE, backprojection adjoint, network backward).  About 0.3 GB on
the device, so `ncu --set full -k regex:<kernel> -s 1 -c 1` on it ends in seconds.

  python -m fdk_b200.profile_learned [n_steps]
"""
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import torch  # noqa: E402

from fdk_b200 import learned as Lr  # noqa: E402

n_steps = int(sys.argv[1]) if len(sys.argv) > 1 else 3
pl = Lr.Pipeline()
p = pl.p
x = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device=pl.dev)
pl.scan(1000, x)
w = torch.from_numpy(Lr.init_params()).to(pl.dev)
w[-(32 * 9 + 1):] = 0.01
torch.cuda.synchronize()
t0 = time.perf_counter()
for _ in range(n_steps):
    pl.truth_of(1000)
    pl.reconstruct(w, x)
    e = pl.mse(True)
    pl.gradient(w, x)
torch.cuda.synchronize()
print(f"{n_steps} steps, {1e3 * (time.perf_counter() - t0) / n_steps:.1f} ms/step, mse {e:.4e}")
