#!/usr/bin/env python
"""FDK reconstruction benchmark: GUPS at 2048^3 x 4096 views of 2048^2 on B200.

One step = one batch of 32 views through the hot path (the workload streams 32-view batches):
cosine weight + ramp/Hann filter at once, backprojection into the resident volume in batches of
512 views (16 steps; a full batch runs when the next one starts, the last two at the final
flush), 128 steps = the whole 4096-view reconstruction.
GUPS = nx*ny*nz*views / seconds / 1e9 (the reference's definition, cuFDK/mpiFDK.h:211,
cudaBP/cudaBP.cpp:68).

  python bench.py [--gpus N --steps K --warmup W] [--precision mixed|fp32|fp32_exact]
  python bench.py --impl reference ...   (the reference's own CPU FDK, 3dct, on host cores)

Under torchrun (N > 1) each rank reconstructs one mirror slab pair of the volume (DivVolume,
cuFDK/mpiFDK.h:116-149); every rank filters all views itself, so there is no collective on
the data path.  Times are device times (CUDA events) and the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GIB = 1 << 30


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- reference arm
def ref_cpu_rate(param, n_views: int, seed: int = 3, slab: int | None = None, log=print) -> dict:
    """Time the reference's own CPU FDK (3dct BackProjection<float>: cosine weight, Bourke FFT
    filter, SSE backprojection; oracle/_ref/libref_cpu.so) on a z-slab of the workload's
    geometry and extrapolate to the full volume: per view, t = t_filter + (nz/slab) * t_bp."""
    from oracle import oracle as O
    import fdk_b200.phantom as P

    cores = os.cpu_count() or 1
    R = O.RefCPU()
    S = slab or max(64, 2 * cores)
    S = min(S, param.nz)
    import copy

    sp = copy.copy(param)
    sp.nz = S
    sp.nProj = param.nProj
    ell = P.phantom_for(param, seed, 30)
    # views of the full-size geometry (the slab sits at the volume centre: same per-voxel cost)
    views = np.stack([O.ellipsoid_projection(ell, param, a) for a in O.view_angles(param)[:n_views]])
    # filter alone (cos weight + Bourke filter rows), as inside BackProjection
    H = O.filter_design(param.str_filter, param.nu)
    cos = O.cos_table(param)
    t0 = time.perf_counter()
    R.filter_rows(H, views[0] * cos * O.angular_ramp_factor(param))
    t_filter = time.perf_counter() - t0
    h = R.fdk_handle(sp, param.str_filter)  # Parameter::init and buffers outside the timing
    try:
        t0 = time.perf_counter()
        R.fdk_run(h, views, 0, threads=cores)
        t_all = time.perf_counter() - t0
    finally:
        R.fdk_destroy(h)
    t_view = t_all / n_views
    t_bp = max(t_view - t_filter, 1e-9)
    t_full = t_filter + t_bp * (param.nz / S)
    gups_full = param.nx * param.ny * param.nz / t_full / 1e9
    gups_sample = param.nx * param.ny * S / t_view / 1e9
    return {"value": gups_full, "sample_gups": gups_sample, "cores": cores, "slab": S, "views": n_views,
            "t_view_s": t_view, "t_filter_s": t_filter, "seconds": t_all}


def run_reference(args, param, rank: int) -> None:
    if rank != 0:
        return
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")
    if not os.path.exists(ref_lib):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref absent"}))
        return
    # calibrate the slab so one step (one view) takes about a second
    cal = ref_cpu_rate(param, 1)
    cores = cal["cores"]
    per_slice = max(cal["t_view_s"] - cal["t_filter_s"], 1e-6) / cal["slab"]
    S = int(max(cores, min(param.nz, (1.0 - min(cal["t_filter_s"], 0.5)) / per_slice)))
    S = max(8, (S // 8) * 8)
    vals, secs = [], 0.0
    for i in range(args.warmup + args.steps):
        r = ref_cpu_rate(param, 1, seed=3 + i, slab=S)
        if i >= args.warmup:
            vals.append(r["value"])
            secs += r["seconds"]
    value = float(np.mean(vals))
    sample = f"{S}-slice z-slab of {param.nx}x{param.ny}, 1 view per step, extrapolated to {param.nz} slices"
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(1, args.steps),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random ellipsoids, exact line integrals)",
        "config": workload_config(param, args),
        "cpu_baseline": {"value": value, "unit": "GUPS", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------- our arm
PUSH = 32    # views per step (one filter launch)
BATCH = 512  # views per backprojection batch (every 16th step); --bp-batch changes it
METRIC = "FDK GUPS at 2048^3 x 4096 views on 1 B200 (mixed precision, rel-L2 <= 1e-3)"


def count_bp_batches(firsts, n: int, batch: int | None = None) -> int:
    """Backprojection batches the reconstructor runs for pushes of n views starting at `firsts`
    (from an empty batch, flushed at the end): one per full batch, per push that does not
    continue the waiting batch, and the final flush.  A batch is one kernel launch per z band.
    batch: views per batch (default: BATCH)."""
    batch = batch or BATCH
    pending, pf, launches = 0, 0, 0
    for f in firsts:
        if pending and f != pf + pending:
            launches, pending = launches + 1, 0
        done = 0
        while done < n:
            if pending == 0:
                pf = f + done
            m = min(n - done, batch - pending)
            pending, done = pending + m, done + m
            if pending == batch:
                launches, pending = launches + 1, 0
    return launches + (1 if pending else 0)


def workload_config(param, args) -> dict:
    return {"workload": f"FDK {param.nx}x{param.ny}x{param.nz} volume from {param.nProj} views of "
                        f"{param.nu}x{param.nv}, batches of {PUSH} views",
            "volume": [param.nx, param.ny, param.nz], "views": param.nProj, "detector": [param.nu, param.nv],
            "batch": PUSH, "bp_batch": BATCH, "precision": args.precision, "filter": param.str_filter,
            "l2": f"inputs larger than L2 ({PUSH * param.nu * param.nv * 4 >> 20} MiB views per step, "
                  f"{param.nx * param.ny * param.nz * 4 >> 30} GiB volume)",
            "parallelism": f"z-slab pairs x{args.gpus}"}


def read_traffic(name: str, key: str):
    """DRAM bytes recorded from an ncu capture: the value of line '<key>: X' in profiles/<name>.md
    (e.g. dram_bytes_per_256_view_batch_full), or None."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(rf"{key}:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def run_ours(args, param, rank: int, world: int, local: int) -> None:
    import torch

    import fdk_b200 as F
    from fdk_b200 import phantom as P
    from fdk_b200.shard import div_volume

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sp = div_volume(param.nx, param.ny, param.nz, rank, world)
    slab = (int(sp.top.z), int(sp.top.depth))
    B = PUSH
    total_batches = args.warmup + args.steps
    n_dev_views = min(param.nProj, B * total_batches)
    frame = param.nu * param.nv
    log = (lambda *a: print(*a, file=sys.stderr, flush=True)) if rank == 0 else (lambda *a: None)

    peaks = F._lib.probe_peaks(local)
    log(f"probes: {peaks}")
    # ---- inputs resident in HBM: exact projections of the seeded phantom
    ell = P.phantom_for(param, 3, 30)
    views = torch.empty((n_dev_views, param.nv, param.nu), dtype=torch.float32, device="cuda")
    for c in range(0, n_dev_views, 256):
        n = min(256, n_dev_views - c)
        P.project(param, ell, c, n, views[c:].data_ptr())
    torch.cuda.synchronize()
    log(f"generated {n_dev_views} views ({n_dev_views * frame * 4 / GIB:.1f} GiB) in HBM")

    def batch_of(b):
        first = (b * B) % param.nProj
        idx = (b * B) % n_dev_views
        return views[idx:idx + B].data_ptr(), first

    def timed_device_run(precision: str, steps: int, warmup: int):
        r = F.Reconstructor(param, precision, batch=BATCH, device=local, slab=slab)
        for b in range(warmup):
            ptr, first = batch_of(b)
            r.push_device(ptr, first, B)
        r.sync()
        st0 = r.stats()
        l0 = r.launch_count
        barrier()
        stream = torch.cuda.ExternalStream(r.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for b in range(warmup, warmup + steps):
            ptr, first = batch_of(b)
            r.push_device(ptr, first, B)
        r.flush()  # backproject a last partial batch inside the timed region
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        barrier()
        st1 = r.stats()
        return r, ms, st1["bp_ms"] - st0["bp_ms"], st1["filter_ms"] - st0["filter_ms"], r.launch_count - l0

    upd_step_all = param.nx * param.ny * param.nz * B          # whole volume, all ranks
    upd_step_rank = param.nx * param.ny * 2 * slab[1] * B      # this rank's slab pair
    clocks = ClockSampler(local)
    clocks.start()
    r, ms, bp_ms, flt_ms, n_launches = timed_device_run(args.precision, args.steps, args.warmup)
    filter_kind = r.filter_kind
    clk = clocks.stop()
    ms_max = allmax(ms)
    n_bp_batches = count_bp_batches([batch_of(b)[1] for b in range(args.warmup, args.warmup + args.steps)], B)
    value = upd_step_all * args.steps / (ms_max * 1e-3) / 1e9
    kernel_gups = upd_step_rank * args.steps / (bp_ms * 1e-3) / 1e9
    log(f"{args.precision}: {ms / args.steps:.2f} ms/step, {value:.1f} GUPS (BP kernels {kernel_gups:.1f} GUPS, "
        f"filter {flt_ms / args.steps:.3f} ms/step), clocks {clk}")

    # ---- accuracy at full size: this precision vs FP32 on a 2x64-slice slab pair, 64 views
    acc = None
    if not args.no_compare and rank == 0 and args.precision != "fp32":
        z0 = slab[0] + max(0, slab[1] // 2 - 32)
        d = min(64, slab[1])
        vols = {}
        for prec in (args.precision, "fp32"):
            ra = F.Reconstructor(param, prec, batch=64, device=local, slab=(z0, d))  # 64 views
            ra.push_device(views.data_ptr(), 0, min(64, n_dev_views))
            vols[prec] = ra.volume().astype(np.float64)
            ra.close()
        a, b = vols[args.precision], vols["fp32"]
        acc = {"vs": "fp32 (staged) on a 128-slice slab pair, 64 views",
               "rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
               "max_abs_rel": float(np.abs(a - b).max() / np.abs(b).max())}
        log(f"accuracy: {acc}")

    # ---- plain FP32 comparison (same workload, fewer steps)
    fp32 = None
    if not args.no_compare and args.precision == "mixed":
        r.close()
        del r
        torch.cuda.empty_cache()
        ks = max(4, args.steps // 8)
        r2, ms2, bp2, _, _ = timed_device_run("fp32", ks, 2)
        v2 = upd_step_all * ks / (allmax(ms2) * 1e-3) / 1e9
        fp32 = {"value": v2, "unit": "GUPS", "steps": ks, "bp_kernel_gups": upd_step_rank * ks / (bp2 * 1e-3) / 1e9,
                "speedup_mixed_over_fp32": value / v2}
        log(f"fp32: {fp32}")
        r2.close()
        del r2
    else:
        r.close()
        del r
    torch.cuda.empty_cache()

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        import psutil

        vol_bytes = param.nx * param.ny * 2 * slab[1] * 4
        avail = psutil.virtual_memory().available / max(1, world)
        pool = int(min(n_dev_views, max(64, (avail * 0.6 - vol_bytes) // (frame * 4))))
        pool = max(B, (pool // B) * B)
        host_views = torch.empty((pool, param.nv, param.nu), dtype=torch.float32, pin_memory=True)
        host_views.copy_(views[:pool])
        host_vol = None
        if avail * 0.8 > vol_bytes + pool * frame * 4:
            host_vol = torch.empty(param.nx * param.ny * 2 * slab[1], dtype=torch.float32, pin_memory=True)
        del views
        torch.cuda.empty_cache()
        re = F.Reconstructor(param, args.precision, batch=BATCH, device=local, slab=slab)
        for b in range(args.warmup):
            re.push_ptr(host_views[(b * B) % pool:].data_ptr(), (b * B) % param.nProj, B)
        re.sync()
        re.reset()
        barrier()
        t0 = time.perf_counter()
        for b in range(args.steps):
            re.push_ptr(host_views[(b * B) % pool:].data_ptr(), (b * B) % param.nProj, B)
        if host_vol is not None:
            re.volume_into(host_vol.data_ptr())
        else:
            re.sync()
        barrier()
        te = allmax(time.perf_counter() - t0)
        e2e = {"value": upd_step_all * args.steps / te / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": B * frame * 4,
               "d2h_bytes_per_step": (vol_bytes // args.steps) if host_vol is not None else 4,
               "seconds": te, "host_pool_views": pool,
               "note": "host views are a pinned pool of the workload's views reused cyclically"
                       if pool < param.nProj else "all views from pinned host memory"}
        log(f"e2e: {e2e}")
        re.close()

    # ---- CPU baseline: the reference's own CPU FDK on a bounded sample (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(
            os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")):
        c = ref_cpu_rate(param, 2)
        cpu = {"value": c["value"], "unit": "GUPS", "cores": c["cores"], "kind": "reference",
               "sample": f"2 views over a {c['slab']}-slice z-slab of {param.nx}x{param.ny} (3dct CPU FDK incl. "
                         f"filtering), extrapolated to {param.nz} slices"}
        log(f"cpu: {c}")

    if rank == 0:
        bpu = 8 if args.precision == "mixed" else 16        # algorithmic shared-memory bytes per update
        fpu = 2 if args.precision == "mixed" else 4         # FMA-pipe operations per update
        peak_smem = peaks["smem_gbs"] * 1e9 / bpu / 1e9
        peak_fma = peaks["fp32_tflops"] * 1e12 / 2 / fpu / 1e9
        peak = min(peak_smem, peak_fma)
        hbm_bytes_batch = (param.nx * param.ny * 2 * slab[1] * (16 if args.precision == "mixed" else 8)
                            + BATCH * frame * (4 if args.precision == "mixed" else 8))
        mp = {}
        try:
            mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
            hbm_peak, hbm_src = mp["hbm_gbs"], "measured"
        except Exception:
            hbm_peak, hbm_src = 6650.0, "fallback"
        bp_batch_ms = bp_ms / n_bp_batches
        bands = (n_launches - args.steps * (2 if filter_kind == "tensor" else 1)) / n_bp_batches
        traffic = read_traffic(f"bp_tma_{args.precision}_c2.md", f"dram_bytes_per_{BATCH}_view_batch_full")
        roofline = {
            "kernel": f"bp_tma_kernel<{'__half2' if args.precision == 'mixed' else 'float2'}>"
            if args.precision != "fp32_exact" else "bp_exact_kernel",
            "bound": "smem" if peak_smem <= peak_fma else "fp32",
            "achieved": kernel_gups, "peak": peak, "unit": "GUPS", "frac": kernel_gups / peak,
            "traffic": traffic,
            "peak_source": (f"measured on this GPU by fdk_probe_smem ({peaks['smem_gbs']:.0f} GB/s) / {bpu} B "
                            f"per update and fdk_probe_fma ({peaks['fp32_tflops']:.1f} TFLOP/s) / {fpu} FMA per "
                            "update"),
            "batch_ms": bp_batch_ms,
            "batch": f"{BATCH} views over the whole volume, run as {bands:g} launches over z bands",
            "hbm": {"achieved": hbm_bytes_batch / (bp_batch_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_bytes_batch / (bp_batch_ms * 1e-3) / 1e9 / hbm_peak, "peak_source": hbm_src,
                    "algorithmic_bytes_per_batch": hbm_bytes_batch},
        }
        out_b = 4 if args.precision == "mixed" else 8
        flt_bytes = B * frame * (4 + out_b)
        flt_step_ms = flt_ms / args.steps
        if filter_kind == "tensor":
            # split FP16: three nu x nu products per row (x_hi M_hi, x_lo M_hi, x_hi M_lo)
            flops = 3 * 2.0 * B * param.nv * param.nu * param.nu
            try:
                tc_peak, tc_src = mp["bf16_tflops_sustained"], "measured (cuBLAS bf16, sustained)"
            except Exception:
                tc_peak, tc_src = 1400.0, "fallback (sustained)"
            filter_roof = {"kernel": "toeplitz_gemm_kernel<f16> (tcgen05; + the weighting pass)",
                           "bound": "tensor", "achieved": flops / (flt_step_ms * 1e-3) / 1e12, "peak": tc_peak,
                           "unit": "TFLOP/s", "frac": flops / (flt_step_ms * 1e-3) / 1e12 / tc_peak,
                           "peak_source": tc_src, "algorithmic_flops_per_step": flops, "launch_ms": flt_step_ms,
                           "hbm_view_gbs": flt_bytes / (flt_step_ms * 1e-3) / 1e9, "traffic": None}
        else:
            filter_roof = {"kernel": "filter_mirror_kernel", "bound": "hbm",
                           "achieved": flt_bytes / (flt_step_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                           "frac": flt_bytes / (flt_step_ms * 1e-3) / 1e9 / hbm_peak,
                           "algorithmic_bytes_per_launch": flt_bytes, "launch_ms": flt_step_ms,
                           "traffic": read_traffic(f"filter_{args.precision}_c2.md", "dram_bytes_per_launch_full")}
        out = {
            "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f16" if args.precision == "mixed" else "f32",
            "data": "synthetic: exact line integrals of a seeded 30-ellipsoid phantom (seed 3)",
            "config": workload_config(param, args),
            "roofline": roofline, "filter_roofline": filter_roof,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": n_launches,
            "filter": filter_kind,
            "plain_fp32": fp32, "accuracy": acc,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    global BATCH
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=128)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp32_exact"])
    ap.add_argument("--config", default="c3")
    ap.add_argument("--bp-batch", type=int, default=BATCH, help="views per backprojection batch")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    BATCH = args.bp_batch
    from fdk_b200.geometry import config

    param = config(args.config)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, param, rank)
    else:
        run_ours(args, param, rank, world, local)


if __name__ == "__main__":
    main()
