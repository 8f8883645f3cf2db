"""Profiling driver: a few filter + backprojection launches at the 512^3 / 512 x 512 x 512-view
configuration (views and volume larger than L2, a few GB on the device), small enough for
`ncu --set full -k regex:bp_ -s 1 -c 1`.

  python -m fdk_b200.profile_bp [mixed|fp32|fp32_exact] [n_batches] [batch]
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import torch  # noqa: E402

import fdk_b200 as F  # noqa: E402
from fdk_b200 import phantom as P  # noqa: E402

prec = sys.argv[1] if len(sys.argv) > 1 else "mixed"
nb = int(sys.argv[2]) if len(sys.argv) > 2 else 3
B = int(sys.argv[3]) if len(sys.argv) > 3 else 128
p = F.config("c2")
p.nProj = max(p.nProj, B * nb)  # views over the full circle; more when the run asks for more
views = torch.empty((B * nb, p.nv, p.nu), dtype=torch.float32, device="cuda")
P.project(p, P.phantom_for(p, 2, 20), 0, B * nb, views.data_ptr())
r = F.Reconstructor(p, prec, batch=B)
for b in range(nb):
    r.push_device(views[B * b:].data_ptr(), B * b, B)
r.sync()
print(prec, r.stats())
