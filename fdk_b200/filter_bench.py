"""Filter variant sweep (the C4 workload by default: 1024 views of 1536 x 1024, W = 2048): the
batched FFT filter against the tensor-core Toeplitz GEMM with FP16 and BF16 operands, plain and
split (hi + lo parts, three products).  Reports
per variant the time per batch of views (CUDA events, inputs resident in HBM), HBM GB/s of the
algorithmic bytes, GEMM TFLOP/s, and rel-L2 / max error of the filtered rows against the FP64
oracle on the first view.  One JSON line.

  python -m fdk_b200.filter_bench [c4|c3] [batch] [reps] [variant,...]

The optional last argument keeps only the named variants (fft, toeplitz_f16, toeplitz_bf16,
toeplitz_f16_split, toeplitz_bf16_split), e.g. to profile one kernel.
"""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import numpy as np  # noqa: E402
import torch  # noqa: E402

import fdk_b200 as F  # noqa: E402
from fdk_b200 import phantom as P  # noqa: E402


def main():
    cfg = sys.argv[1] if len(sys.argv) > 1 else "c4"
    batch = int(sys.argv[2]) if len(sys.argv) > 2 else 128
    reps = int(sys.argv[3]) if len(sys.argv) > 3 else 5
    only = set(sys.argv[4].split(",")) if len(sys.argv) > 4 else None
    keep = lambda name: only is None or name in only  # noqa: E731
    p = F.config(cfg)
    nu, nv = p.nu, p.nv
    s = float(1.0 / (p.SOD * p.SOD * p.AngularAndrampFactor))
    views = torch.empty((batch, nv, nu), dtype=torch.float32, device="cuda")
    P.project(p, P.phantom_for(p, 4, 20), 0, batch, views.data_ptr())
    out = torch.empty((batch, nu, nv, 2), dtype=torch.float16, device="cuda")
    frame = nu * nv
    W = int(F.lib().fdk_filter_length(nu))
    res = {"workload": f"{cfg}: {batch} views of {nu}x{nv} per batch, W = {W}", "variants": {}}

    def timed(run):
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    # reference rows of view 0 (FP64 oracle) in line-integral units
    from oracle import oracle as O
    v0 = views[0].cpu().numpy()
    want = O.filter_view(v0, O.filter_design(p.str_filter, nu), O.cos_table(p), pad_n=4, transpose=True) * s

    def errors(mirror):
        got = mirror[0, :, :, 0].float().cpu().numpy()  # (nu, nv): element (u, v) main row
        return {"rel_l2": float(np.linalg.norm(got - want) / np.linalg.norm(want)),
                "max_rel": float(np.abs(got - want).max() / np.abs(want).max())}

    if keep("fft"):
        eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32, pad_edge=4)
        ms = timed(lambda: eng.run_device(views.data_ptr(), out.data_ptr(), batch, F.LAYOUT_MIRROR, F.DTYPE_F16, s))
        hbm = batch * frame * (4 + 4)
        res["variants"]["fft"] = {"ms": ms, "hbm_gbs": hbm / (ms * 1e-3) / 1e9, **errors(out)}
    flops = 2.0 * batch * nv * nu * nu
    for dt, split in (("f16", False), ("bf16", False), ("f16", True), ("bf16", True)):
        name = f"toeplitz_{dt}{'_split' if split else ''}"
        if not keep(name):
            continue
        tf = F.ToeplitzFilter(p.cos_sigma, p.fft_kernel_real, 4, dt, in_scale=s, split=split)
        ms = timed(lambda: tf.run_device(views.data_ptr(), out.data_ptr(), batch, F.LAYOUT_MIRROR, 1.0))
        tf.check()
        terms = 3 if split else 1
        res["variants"][name] = {
            "ms": ms, "tflops": terms * flops / (ms * 1e-3) / 1e12, **errors(out)}
        tf.close()
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
