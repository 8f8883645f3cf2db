#!/usr/bin/env python
"""FDK reconstruction benchmark: GUPS at 2048^3 x 4096 views of 2048^2 on B200.

One step = one batch of 32 views through the hot path (the workload streams 32-view batches):
cosine weight + ramp/Hann filter at once, backprojection into the resident volume in batches of
512 views (a full batch runs when the next one starts, the last two at the final flush), 128
steps = the whole 4096-view reconstruction.
GUPS = nx*ny*nz*views / seconds / 1e9 (the reference's definition, cuFDK/mpiFDK.h:211,
cudaBP/cudaBP.cpp:68).

  python bench.py [--gpus N --steps K --warmup W] [--precision mixed|fp32|fp32_exact] [--config c3]
  python bench.py --impl reference ...   (the reference's own CPU FDK, 3dct, on host cores)
  python bench.py --kernel bp|filter|rtk|learned ...   (one kernel family on a small case, for
                                                         ncu captures and tuning sweeps)

Besides `value` (device time, views resident in HBM) and `e2e` (host buffers through
fdk_recon_push, the volume back to pinned host memory), the line carries:
  accuracy      the run's views reconstructed at full size in MIXED and FP32, checked against
                the FP64 oracle at sampled voxels and the central x, y, z slices; FP32 (staged)
                against the reference kernel's arithmetic (fp32_exact) on a central slab pair
  plain_fp32    the same timed run in plain FP32
  reference_gpu the reference's own cudaFdkBP (compiled for sm_100a) on a 2048^2 x 512 slab
                pair beside ours on the same views
  cpu_baseline  the reference's CPU FDK (3dct) timed on the host cores, extrapolated per view
  roofline      the backprojection kernel against its measured shared-memory roofline

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
        return parse_clock_lines(self.lines)


def parse_clock_lines(lines) -> dict:
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
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


# --------------------------------------------------------------------------- reference CPU FDK
def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class RefCpuTimer:
    """The reference's own CPU FDK (3dct BackProjection<float>: cosine weight, Bourke FFT filter,
    SSE backprojection; oracle/_ref/libref_cpu.so) on all host cores, timed on z-slabs of the
    workload's geometry centred in the volume (the same per-voxel work as the whole volume).

    Per view the reference's cost is t(S) = f + b*S for an S-slice slab: f is the filtering and
    per-view set-up, b one slice of backprojection.  calibrate() times `repeats` passes of the
    same `views` views at S and at S/2 (medians) and one pass at S/4 as a linearity check; the
    whole volume then costs f + b*nz per view.  Used by the cpu_baseline leg and by
    --impl reference alike, so both report the same quantity."""

    def __init__(self, param, views: int = 4, slab: int = 256, seed: int = 3, threads: int = 0):
        from oracle import oracle as O
        import copy

        import fdk_b200.phantom as P

        self.O, self.param = O, param
        self.R = O.RefCPU()
        self.cores = threads or os.cpu_count() or 1
        self.n_views = views
        self.S = min(param.nz, slab)
        ell = P.phantom_for(param, seed, 30)
        angles = O.view_angles(param)
        self.views = np.stack([O.ellipsoid_projection(ell, param, angles[i]) for i in range(views)])
        self.handles = {}
        for S in sorted({self.S, max(1, self.S // 2), max(1, self.S // 4)}):
            sp = copy.copy(param)
            sp.nz = S
            self.handles[S] = self.R.fdk_handle(sp, param.str_filter)  # tables and buffers, untimed
        self.f = self.b = None
        self.calib = {}

    def run(self, S: int) -> float:
        """Seconds for one pass of the views through 3dct over an S-slice slab."""
        t0 = time.perf_counter()
        self.R.fdk_run(self.handles[S], self.views, 0, threads=self.cores)
        return time.perf_counter() - t0

    def calibrate(self, repeats: int = 3) -> dict:
        S, h = self.S, max(1, self.S // 2)
        self.run(S)  # warm-up (page faults of the slab buffers)
        tS = [self.run(S) for _ in range(repeats)]
        th = [self.run(h) for _ in range(repeats)] if h < S else tS
        mS, mh = statistics.median(tS), statistics.median(th)
        V = self.n_views
        if h < S:
            self.b = max((mS - mh) / V / (S - h), 1e-12)
            self.f = max(mS / V - self.b * S, 0.0)
        else:  # the slab is the whole volume
            self.b, self.f = mS / V / S, 0.0
        q = max(1, S // 4)
        t4 = self.run(q) if q < h else None
        self.calib = {"slab_s": [S, h], "t_pass_s": {str(S): tS, str(h): th}, "f_view_s": self.f,
                      "b_slice_s": self.b,
                      "linearity": (None if t4 is None else
                                    {"slices": q, "measured_s": t4, "predicted_s": V * (self.f + self.b * q)}),
                      "gups_spread": [self.gups(t, S) for t in (max(tS), min(tS))]}
        return self.calib

    def gups(self, t_pass: float, S: int) -> float:
        """Whole-volume GUPS implied by one pass over an S-slice slab taking t_pass seconds."""
        p = self.param
        per_view = t_pass / self.n_views
        if self.f is not None and S < p.nz:
            per_view *= (self.f + self.b * p.nz) / (self.f + self.b * S)
        return p.nx * p.ny * p.nz / per_view / 1e9

    def sample_text(self) -> str:
        p = self.param
        return (f"{self.n_views} views through 3dct over a {self.S}-slice z-slab of {p.nx}x{p.ny} (median of 3 passes), "
                f"extrapolated to {p.nz} slices per view as f + b*nz (f, b from slabs of {self.S} and "
                f"{max(1, self.S // 2)} slices); {self.cores} threads on {cpu_model()}")

    def close(self):
        for h in self.handles.values():
            self.R.fdk_destroy(h)
        self.handles = {}


def ref_cpu_full(param, threads: int = 0) -> dict:
    """The reference's CPU FDK over the whole volume and every view (the small workloads run in
    full): all views projected, then one timed run of 3dct."""
    from oracle import oracle as O

    import fdk_b200.phantom as P

    R = O.RefCPU()
    cores = threads or os.cpu_count() or 1
    n_ell = 20 if param.nx <= 512 else 30
    ell = P.phantom_for(param, 2, n_ell)
    views = np.stack([O.ellipsoid_projection(ell, param, a) for a in O.view_angles(param)])
    h = R.fdk_handle(param, param.str_filter)
    try:
        t0 = time.perf_counter()
        R.fdk_run(h, views, 0, threads=cores)
        t = time.perf_counter() - t0
    finally:
        R.fdk_destroy(h)
    return {"value": param.nx * param.ny * param.nz * param.nProj / t / 1e9, "unit": "GUPS", "seconds": t,
            "cores": cores, "cpu": cpu_model(), "sample": "whole volume, every view"}


def run_reference(args, param, rank: int) -> None:
    if rank != 0:
        return
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")
    if not os.path.exists(ref_lib):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref absent"}))
        return
    T = RefCpuTimer(param)
    cal = T.calibrate()
    vals, secs = [], 0.0
    for i in range(args.warmup + args.steps):
        t = T.run(T.S)
        if i >= args.warmup:
            vals.append(T.gups(t, T.S))
            secs += t
    T.close()
    value = float(statistics.median(vals))
    out = {
        "impl": "reference", "metric": metric_name(param, args.precision), "value": value, "unit": "GUPS", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(1, args.steps),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random ellipsoids, exact line integrals)",
        "config": workload_config(param, args),
        "cpu_baseline": {"value": value, "unit": "GUPS", "cores": T.cores, "kind": "reference",
                         "sample": "each step: " + T.sample_text(), "spread": [min(vals), max(vals)],
                         "calibration": cal},
        "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------- our arm
PUSH = 32    # views per step (one filter launch)
BATCH = 512  # views per backprojection batch (every 16th step); --bp-batch changes it
METRIC = "FDK GUPS at 2048^3 x 4096 views on 1 B200 (mixed precision, rel-L2 <= 1e-3)"
L2_BYTES = 126 << 20


def metric_name(param, precision: str) -> str:
    """The headline metric for the 2048^3 / 4096-view MIXED workload; the same wording with the
    workload's own sizes and precision otherwise."""
    if (param.nx, param.ny, param.nz, param.nProj) == (2048, 2048, 2048, 4096) and precision == "mixed":
        return METRIC
    shape = f"{param.nx}^3" if param.nx == param.ny == param.nz else f"{param.nx}x{param.ny}x{param.nz}"
    prec = "mixed precision, rel-L2 <= 1e-3" if precision == "mixed" else f"{precision} precision"
    return f"FDK GUPS at {shape} x {param.nProj} views on 1 B200 ({prec})"


READ_ORDER = "quarter"  # set by main(): "quarter" or "sequential"


def step_chunks(param, b: int, B: int = PUSH, order: str | None = None) -> list:
    """The views of step b as (first, count) chunks.  Quarter order: B/4 consecutive views from
    each quarter of the scan (view v + k N/4, k = 0..3), in which every batch holds whole
    quarter-turn quadruples (fdk_recon_bp_kernel); all 128 steps of the 4096-view scan read each
    view once.  Sequential order, and scans whose quarter is not a multiple of B/4 views: B
    consecutive views."""
    N = param.nProj
    c = B // 4
    if (order or READ_ORDER) == "quarter" and B % 4 == 0 and N % 4 == 0 and (N // 4) % c == 0:
        q = N // 4
        base = (b * c) % q
        return [(base + k * q, c) for k in range(4)]
    return [((b * B) % N, B)]


def count_bp_batches(firsts, n: int, batch: int | None = None, contiguous: bool = False) -> list:
    """Sizes of the backprojection batches the reconstructor runs for pushes of n views
    starting at `firsts` (from an empty batch, flushed at the end): one per full batch and the
    final flush; with `contiguous` (FP32_EXACT) also one per push that does not continue the
    waiting batch.  batch: views per batch (default: BATCH)."""
    batch = batch or BATCH
    sizes = []
    pending, pf = 0, 0
    for f in firsts:
        if contiguous and pending and f != pf + pending:
            sizes.append(pending)
            pending = 0
        done = 0
        while done < n:
            if pending == 0:
                pf = f + done
            m = min(n - done, batch - pending)
            pending, done = pending + m, done + m
            if pending == batch:
                sizes.append(pending)
                pending = 0
    if pending:
        sizes.append(pending)
    return sizes


def conversion_launches(precision: str) -> int:
    """Launches a backprojection batch makes before its bands: MIXED finds the batch's largest
    magnitude and converts its views to the interpolation layout."""
    return 2 if precision == "mixed" else 0


def band_launches(n_launches: int, steps: int, filter_per_step: int, n_batches: int, precision: str) -> float:
    """Band launches per backprojection batch, from the library's launch count of a timed run:
    each step's filter launches and each batch's conversion launches taken out."""
    return (n_launches - steps * filter_per_step) / max(1, n_batches) - conversion_launches(precision)


def l2_note(param, precision: str) -> str:
    """How the timed steps stand to the 126 MB L2: the volume (and the MIXED compensation) is
    read and written by every batch, so it decides whether a step can hit L2."""
    views = PUSH * param.nu * param.nv * 4
    vol = param.nx * param.ny * param.nz * 4 * (2 if precision == "mixed" else 1)
    sizes = f"{views / 2**20:.0f} MiB views per step, {vol / 2**20:.0f} MiB volume state"
    if vol > L2_BYTES:
        return f"inputs larger than L2 ({sizes})"
    return f"inputs smaller than L2 ({sizes}): L2 not flushed between steps"


def workload_config(param, args) -> dict:
    return {"workload": f"FDK {param.nx}x{param.ny}x{param.nz} volume from {param.nProj} views of "
                        f"{param.nu}x{param.nv}, batches of {PUSH} views",
            "volume": [param.nx, param.ny, param.nz], "views": param.nProj, "detector": [param.nu, param.nv],
            "batch": PUSH, "bp_batch": BATCH, "precision": args.precision, "filter": param.str_filter,
            "l2": l2_note(param, args.precision),
            "parallelism": f"z-slab pairs x{args.gpus}"}


def read_traffic(name: str, key: str):
    """DRAM bytes recorded from an ncu capture: the value of line '<key>: X' in profiles/<name>.md
    (e.g. dram_bytes_per_512_view_batch_full), or None."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(rf"{key}:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def errors(got: np.ndarray, want: np.ndarray, mask=None) -> dict:
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    out = {"rel_l2": float(np.linalg.norm(got - want) / np.linalg.norm(want)),
           "max_abs_rel": float(np.abs(got - want).max() / np.abs(want).max()), "voxels": int(got.size)}
    if mask is not None and mask.any():
        g, w = got[~mask], want[~mask]
        out["masked"] = {"rel_l2": float(np.linalg.norm(g - w) / np.linalg.norm(w)),
                         "max_abs_rel": float(np.abs(g - w).max() / np.abs(w).max()),
                         "excluded_knife_edge_voxels": int(mask.sum())}
    return out


def accuracy_leg(F, param, views, chunks_of, steps: int, slab, local: int, log) -> dict:
    """The run's views (steps 0..steps-1, chunks_of(b) -> (device pointer, view indices)),
    reconstructed at full size in MIXED and FP32, against the FP64 oracle (checker only) at 1e5
    seeded voxels and every voxel of the central x, y and z slices of this rank's slab pair; then
    FP32 (staged) against the reference kernel's arithmetic (fp32_exact, bit-identical to
    cudaFdkBP) on a central 2 x 64-slice slab pair.  Knife-edge voxels (projected within 1e-3 px
    of a detector border in some view, where the reference's bounds rule is discontinuous) are
    reported unmasked and excluded."""
    from oracle import oracle as O

    import torch

    t0 = time.perf_counter()
    vox = O.sample_voxels(param.nx, param.ny, param.nz, 100000, 17)
    z0, d = slab
    inside = ((vox[:, 2] >= z0) & (vox[:, 2] < z0 + d)) | ((vox[:, 2] >= param.nz - z0 - d) &
                                                             (vox[:, 2] < param.nz - z0))
    vox = np.ascontiguousarray(vox[inside])
    pushes = [chunks_of(b) for b in range(steps)]
    got, kind = {}, {}
    for prec in ("mixed", "fp32"):
        r = F.Reconstructor(param, prec, batch=BATCH, device=local, slab=slab)
        for ptr, ids in pushes:
            r.push_device_views(ptr, ids)
        got[prec] = r.sample(vox)
        kind[prec] = r.bp_kernel
        r.close()
    S = O.SampledFDK(param, vox)
    frame = param.nu * param.nv
    for ptr, ids in pushes:
        i = (ptr - views.data_ptr()) // (4 * frame)
        j = 0
        while j < len(ids):  # the oracle takes runs of consecutive views
            k = j + 1
            while k < len(ids) and ids[k] == ids[k - 1] + 1:
                k += 1
            S.add(views[i + j:i + k].cpu().numpy(), int(ids[j]))
            j = k
    mask = S.edge.astype(bool)
    n_views = sum(len(ids) for _, ids in pushes)
    res = {"vs": "fp64 oracle (sampled)", "views": n_views, "bp_kernel": kind,
           "voxels": f"{len(vox)}: 1e5 seeded random voxels + the central x, y and z slices (within the slab pair)",
           "mixed": errors(got["mixed"], S.values, mask), "fp32": errors(got["fp32"], S.values, mask)}
    # FP32 staged against the reference arithmetic on a central slab pair
    zc = z0 + max(0, d // 2 - 32) if z0 + d < param.nz // 2 else max(z0, param.nz // 2 - 64)
    dc = min(64, d)
    vols = {}
    for prec in ("fp32", "fp32_exact"):
        r = F.Reconstructor(param, prec, batch=32 if prec == "fp32_exact" else BATCH, device=local, slab=(zc, dc))
        for ptr, ids in pushes:
            r.push_device_views(ptr, ids)
        vols[prec] = r.volume().astype(np.float64)
        r.close()
    res["fp32_vs_fp32_exact"] = {"slab_pair": [zc, dc], **errors(vols["fp32"], vols["fp32_exact"])}
    res["seconds"] = time.perf_counter() - t0
    torch.cuda.empty_cache()
    log(f"accuracy: {res}")
    return res


def reference_gpu_leg(F, param, views, chunks_of, local: int, log) -> dict | None:
    """The reference's own cudaFdkBP (oracle/_ref/libref_gpu_bp.so, compiled for sm_100a) on the
    per-GPU ABCI shape: a 2048 x 2048 x (2 x 256) slab pair (its 32-bit voxel offsets stay valid)
    from 2048^2 views, 32 views per BP() call, next to our precisions on 128 views of the run
    (in 128-view batches; FP32 and MIXED also with the other kernel choice, FDK_BP_SYM)."""
    from oracle import oracle as O

    import torch

    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_gpu_bp.so")):
        return None
    n = PUSH
    zc, dc = param.nz // 2 - 256, 256
    # filtered views in the reference's transposed layout (nu rows of nv), FP32, from our filter
    eng = F.FilterEngine(param.cos_sigma, param.fft_kernel_real_f32, pad_edge=4)
    filt = torch.empty((n, param.nu, param.nv), dtype=torch.float32, device="cuda")
    eng.run_device(views.data_ptr(), filt.data_ptr(), n, F.LAYOUT_TRANSPOSED, F.DTYPE_F32, 1.0)
    torch.cuda.synchronize()
    host = filt.cpu().numpy()
    del filt
    eng.close()
    mats = param.proj_matrices()[:n]
    top = [0, 0, zc, param.nx, param.ny, dc]
    bot = [0, 0, param.nz - zc - dc, param.nx, param.ny, dc]
    ref = O.RefGPU().time_bp(host, mats, param.nx, param.ny, param.nz, top, bot)
    upd = param.nx * param.ny * 2 * dc * n
    out = {"slab_pair": f"{param.nx}x{param.ny}x(2x{dc}) at z {zc}", "views_per_call": n,
           "reference_kernel_gups": upd / (ref["kernel_ms"] * 1e-3) / 1e9,
           "reference_bp_call_gups": upd / (ref["call_ms"] * 1e-3) / 1e9,
           "reference_note": "BP() call = H2D copy of the views + kernel + cudaDeviceSynchronize (stock path)"}
    ours = {}
    pushes = [chunks_of(b) for b in range(4)]  # 128 views
    # each precision with the reconstructor's default kernel choice, then the other choice
    for prec, sym in (("fp32_exact", None), ("fp32", None), ("mixed", None), ("fp32", "0"), ("mixed", "1")):
        if sym is not None:
            os.environ["FDK_BP_SYM"] = sym
        r = F.Reconstructor(param, prec, batch=32 if prec == "fp32_exact" else 128, device=local, slab=(zc, dc))
        os.environ.pop("FDK_BP_SYM", None)
        r.push_device_views(*pushes[0])  # warm-up
        r.sync()
        r.reset()
        for ptr, ids in pushes:
            r.push_device_views(ptr, ids)
        r.sync()
        st = r.stats()
        key = prec if sym is None else f"{prec}_{r.bp_kernel}"
        ours[key] = {"gups": param.nx * param.ny * 2 * dc * 128 / (st["bp_ms"] * 1e-3) / 1e9, "kernel": r.bp_kernel}
        r.close()
    out["ours"] = ours
    out["ratio_over_reference_kernel"] = {k: v["gups"] / out["reference_kernel_gups"] for k, v in ours.items()}
    torch.cuda.empty_cache()
    log(f"reference_gpu: {out}")
    return out


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
    pool_steps = min(total_batches, max(1, param.nProj // B))  # distinct steps held in HBM
    n_dev_views = pool_steps * B
    frame = param.nu * param.nv
    log = (lambda *a: print(*a, file=sys.stderr, flush=True)) if rank == 0 else (lambda *a: None)

    peaks = F._lib.probe_peaks(local)
    log(f"probes: {peaks}")
    # ---- inputs resident in HBM: exact projections of the seeded phantom, in step order (step
    # b's chunks, step_chunks(), one after another; steps beyond the pool reuse it cyclically).
    # Each leg reads in the order its reconstructor runs best (READ_ORDER for the timed
    # precision); a pool in another order is generated when a leg needs one.
    ell = P.phantom_for(param, 3, 30)
    pools = {}

    def pool(order):
        if order not in pools:
            for k in list(pools):  # one pool at a time on the device
                del pools[k]
            torch.cuda.empty_cache()
            v = torch.empty((n_dev_views, param.nv, param.nu), dtype=torch.float32, device="cuda")
            for b in range(pool_steps):
                o = b * B
                for first, n in step_chunks(param, b, order=order):
                    P.project(param, ell, first, n, v[o:].data_ptr())
                    o += n
            torch.cuda.synchronize()
            pools[order] = v
            log(f"generated {n_dev_views} views ({n_dev_views * frame * 4 / GIB:.1f} GiB, {order} order) in HBM")
        return pools[order]

    def chunks_of(b, order=None):
        """Step b's push: (device pointer of its B views in the pool, their view indices)."""
        order = order or READ_ORDER
        ids = np.array([v for first, n in step_chunks(param, b, order=order) for v in range(first, first + n)],
                       np.int64)
        return pool(order)[(b % pool_steps) * B:].data_ptr(), ids

    def order_of(precision):
        return "quarter" if pairs_views(param, precision) else "sequential"

    def timed_device_run(precision: str, steps: int, warmup: int, order=None):
        order = order or READ_ORDER
        pool(order)
        r = F.Reconstructor(param, precision, batch=BATCH, device=local, slab=slab)
        for b in range(warmup):
            r.push_device_views(*chunks_of(b, order))
        r.sync()
        st0 = r.stats()
        l0 = r.launch_count
        barrier()
        stream = torch.cuda.ExternalStream(r.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for b in range(warmup, warmup + steps):
            r.push_device_views(*chunks_of(b, order))
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
    bp_kind = r.bp_kernel
    clk = clocks.stop()
    r.close()
    del r
    torch.cuda.empty_cache()
    ms_max = allmax(ms)
    pushes = [c for b in range(args.warmup, args.warmup + args.steps) for c in step_chunks(param, b)]
    batch_sizes = count_bp_batches([f for f, _ in pushes], pushes[0][1], contiguous=args.precision == "fp32_exact")
    value = upd_step_all * args.steps / (ms_max * 1e-3) / 1e9
    kernel_gups = upd_step_rank * args.steps / (bp_ms * 1e-3) / 1e9
    log(f"{args.precision}: {ms / args.steps:.2f} ms/step, {value:.1f} GUPS (BP kernels {kernel_gups:.1f} GUPS, "
        f"filter {flt_ms / args.steps:.3f} ms/step), clocks {clk}")

    # ---- plain FP32: the same timed run (same steps and warm-up) in FP32
    fp32 = None
    if not args.no_compare and args.precision == "mixed":
        r2, ms2, bp2, _, _ = timed_device_run("fp32", args.steps, args.warmup, order_of("fp32"))
        fp32_kind = r2.bp_kernel
        r2.close()
        del r2
        torch.cuda.empty_cache()
        v2 = upd_step_all * args.steps / (allmax(ms2) * 1e-3) / 1e9
        fp32 = {"value": v2, "unit": "GUPS", "steps": args.steps, "warmup": args.warmup,
                "bp_kernel_gups": upd_step_rank * args.steps / (bp2 * 1e-3) / 1e9,
                "speedup_mixed_over_fp32": value / v2, "bp_kernel": fp32_kind, "read_order": order_of("fp32")}
        log(f"fp32: {fp32}")

    # ---- accuracy at full size against the FP64 oracle (rank 0; the checker, not timed)
    acc = None
    if not args.no_compare and rank == 0:
        acc = accuracy_leg(F, param, pool("quarter"), lambda b: chunks_of(b, "quarter"), min(args.steps, pool_steps),
                           slab, local, log)

    # ---- the reference's own GPU backprojector beside ours (rank 0, N = 1)
    ref_gpu = None
    if not args.no_compare and rank == 0 and world == 1 and param.nu == 2048 and param.nx == 2048:
        ref_gpu = reference_gpu_leg(F, param, pool("quarter"), lambda b: chunks_of(b, "quarter"), local, log)

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        import psutil

        vol_bytes = param.nx * param.ny * 2 * slab[1] * 4
        avail = psutil.virtual_memory().available / max(1, world)
        pool_n = int(min(n_dev_views, max(64, (avail * 0.6 - vol_bytes) // (frame * 4))))
        pool_n = max(B, (pool_n // B) * B)  # whole steps of the device pool's step order
        host_views = torch.empty((pool_n, param.nv, param.nu), dtype=torch.float32, pin_memory=True)
        host_views.copy_(pool(READ_ORDER)[:pool_n])
        host_vol = None
        if avail * 0.8 > vol_bytes + pool_n * frame * 4:
            host_vol = torch.empty(param.nx * param.ny * 2 * slab[1], dtype=torch.float32, pin_memory=True)
        pools.clear()
        torch.cuda.empty_cache()
        host_steps = pool_n // B

        def host_step(b):
            ids = np.array([v for first, n in step_chunks(param, b % host_steps) for v in range(first, first + n)],
                           np.int64)
            return host_views[(b % host_steps) * B:].data_ptr(), ids

        re = F.Reconstructor(param, args.precision, batch=BATCH, device=local, slab=slab)
        for b in range(args.warmup):
            re.push_views_ptr(*host_step(b))
        re.sync()
        re.reset()
        barrier()
        t0 = time.perf_counter()
        for b in range(args.steps):
            re.push_views_ptr(*host_step(b))
        t_push = time.perf_counter() - t0
        if host_vol is not None:
            re.volume_into(host_vol.data_ptr())
        else:
            re.sync()
        barrier()
        te = allmax(time.perf_counter() - t0)
        e2e = {"value": upd_step_all * args.steps / te / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": B * frame * 4,
               "d2h_bytes_per_step": (vol_bytes // args.steps) if host_vol is not None else 4,
               "seconds": te, "push_seconds": t_push, "host_pool_views": pool_n,
               "note": ("the whole volume is read back once at the end, counted per step; "
                        + ("host views are a pinned pool of the workload's views reused cyclically"
                           if pool_n < param.nProj else "all views from pinned host memory"))}
        log(f"e2e: {e2e}")
        re.close()

    # ---- CPU baseline: the reference's own CPU FDK on a bounded sample (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(
            os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")):
        if args.cpu_full:
            c = ref_cpu_full(param)
            cpu = {**c, "kind": "reference"}
        else:
            T = RefCpuTimer(param)
            cal = T.calibrate()
            T.close()
            cpu = {"value": float(statistics.median([T.gups(t, T.S) for t in cal["t_pass_s"][str(T.S)]])),
                   "unit": "GUPS", "cores": T.cores, "kind": "reference", "sample": T.sample_text(),
                   "spread": cal["gups_spread"], "calibration": cal}
        log(f"cpu: {cpu}")

    if rank == 0:
        bpu = 8 if args.precision == "mixed" else 16        # algorithmic shared-memory bytes per update
        fpu = 2 if args.precision == "mixed" else 4         # FMA-pipe operations per update
        peak_smem = peaks["smem_gbs"] * 1e9 / bpu / 1e9
        peak_fma = peaks["fp32_tflops"] * 1e12 / 2 / fpu / 1e9
        peak = min(peak_smem, peak_fma)
        vol_rmw = param.nx * param.ny * 2 * slab[1] * (16 if args.precision == "mixed" else 8)
        # bytes per view the kernel reads: FP32 mirror pairs, or MIXED's interpolation layout
        # (8 B per element; the FP16 gather of the quarter-turn kernel reads 4)
        view_bytes = frame * (4 if args.precision == "mixed" and bp_kind == "quarter-turn" else 8)
        views_run = sum(batch_sizes)
        hbm_bytes = len(batch_sizes) * vol_rmw + views_run * view_bytes   # all batches of the run
        mp = {}
        try:
            mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
            hbm_peak, hbm_src = mp["hbm_gbs"], "measured"
        except Exception:
            hbm_peak, hbm_src = 6650.0, "fallback"
        conv = conversion_launches(args.precision)
        bands = band_launches(n_launches, args.steps, 2 if filter_kind == "tensor" else 1, len(batch_sizes),
                              args.precision)
        # the staged kernel's DRAM bytes recorded by an ncu capture (MIXED: the interpolation layout)
        traffic = read_traffic("bp_tma_lerp_c2.md" if args.precision == "mixed" else f"bp_tma_{args.precision}_c2.md",
                               f"dram_bytes_per_{BATCH}_view_batch_full")
        if traffic is not None and bp_kind != "staged":
            traffic = None  # the figure is the staged kernel's
        nvox = param.nx * param.ny * param.nz
        if traffic is not None and nvox != 2048 ** 3:
            traffic *= nvox / 2048 ** 3  # recorded for 2048^3 (scaled by voxel count from a 512^3 capture)
        et = '__half2' if args.precision == 'mixed' else 'float2'
        staged = ("bp_tma_kernel<HalfLerp*> (views converted to the interpolation layout; compact boxes where "
                  "every tile fits)" if args.precision == "mixed" else f"bp_tma_kernel<{et}>")
        roofline = {
            "kernel": {"quarter-turn": f"bp_sym_kernel<{et}> (views paired with their quarter-turn partners)",
                       "staged": staged, "exact": "bp_exact_kernel"}[bp_kind],
            "bound": "smem" if peak_smem <= peak_fma else "fp32",
            "achieved": kernel_gups, "peak": peak, "unit": "GUPS", "frac": kernel_gups / peak,
            "traffic": traffic,
            "traffic_unit": f"DRAM bytes per full {BATCH}-view batch of this workload (ncu capture at 512^3, "
                            "scaled by voxel count; see profiles)",
            "peak_source": (f"measured on this GPU by fdk_probe_smem ({peaks['smem_gbs']:.0f} GB/s) / {bpu} B "
                            f"per update and fdk_probe_fma ({peaks['fp32_tflops']:.1f} TFLOP/s) / {fpu} FMA per "
                            "update"),
            "batches": batch_sizes,
            "ms_per_view": bp_ms / views_run,
            "batch": f"batches of up to {BATCH} views over the whole slab pair, each run as {bands:g} launches "
                     "over z bands" + (f" after {conv} view-conversion launches" if conv else ""),
            "hbm": {"achieved": hbm_bytes / (bp_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_bytes / (bp_ms * 1e-3) / 1e9 / hbm_peak, "peak_source": hbm_src,
                    "algorithmic_bytes_of_the_run": hbm_bytes,
                    "per_batch": "volume (+ compensation) read and written once + its views as the kernel "
                                 "reads them"},
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
            "metric": metric_name(param, args.precision), "value": value, "unit": "GUPS", "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f16" if args.precision == "mixed" else "f32",
            "data": "synthetic: exact line integrals of a seeded 30-ellipsoid phantom (seed 3)",
            "config": workload_config(param, args),
            "roofline": roofline, "filter_roofline": filter_roof,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": n_launches,
            "filter": filter_kind, "bp_kernel": bp_kind,
            "read_order": (READ_ORDER + (": each step reads 8 consecutive views from each quarter of the scan "
                                         "(views v + k N/4)" if READ_ORDER == "quarter" else
                                         ": each step reads 32 consecutive views") +
                           "; the 128 steps of the whole scan read every view once"),
            "plain_fp32": fp32, "accuracy": acc, "reference_gpu": ref_gpu,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------- kernel sub-benches
def timed(run, reps: int) -> float:
    import torch

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def kernel_bp(args) -> None:
    """Backprojection batches through the reconstructor on device-resident views (default: the
    512^3 / 512^2 geometry, 3 batches of 128 views read in the bench's quarter order -- views and
    volume larger than L2, a few GB on the device, small enough for
    `ncu --set full -k regex:bp_ -s 1 -c 1`).  --variants staged: without the quarter-turn
    pairing (FDK_BP_SYM=0); --variants paired: with it for MIXED too (FDK_BP_SYM=1)."""
    import torch

    import fdk_b200 as F
    from fdk_b200 import phantom as P

    nb, B = args.batches, args.bp_batch
    p = F.config(args.config)
    p.nProj = max(p.nProj, B * nb)  # views over the full circle; more when the run asks for more
    steps = B * nb // PUSH
    pushes = [c for b in range(steps) for c in step_chunks(p, b, order="quarter")]
    views = torch.empty((B * nb, p.nv, p.nu), dtype=torch.float32, device="cuda")
    ell = P.phantom_for(p, 2, 20)
    o = 0
    for first, n in pushes:
        P.project(p, ell, first, n, views[o:].data_ptr())
        o += n
    if args.variants in ("staged", "paired"):
        os.environ["FDK_BP_SYM"] = "0" if args.variants == "staged" else "1"
    r = F.Reconstructor(p, args.precision, batch=B)
    os.environ.pop("FDK_BP_SYM", None)
    o = 0
    for first, n in pushes:
        r.push_device(views[o:].data_ptr(), first, n)
        o += n
    r.sync()
    st = r.stats()
    st["gups"] = p.nx * p.ny * p.nz * B * nb / (st["bp_ms"] * 1e-3) / 1e9
    print(json.dumps({"kernel": "bp", "config": args.config, "precision": args.precision, "batch": B,
                      "batches": nb, "bp_kernel": r.bp_kernel, **st}), flush=True)
    r.close()


def kernel_filter(args) -> None:
    """Filter variants on device-resident views (default c4: 1536 x 1024, W = 2048): the batched
    FFT filter and the tensor-core Toeplitz GEMM (FP16/BF16, plain and split), time per batch of
    `--bp-batch` views (CUDA events), HBM GB/s of the algorithmic bytes, GEMM TFLOP/s.  Accuracy
    of each variant against the FP64 oracle is checked in tests/test_gpu_toeplitz.py."""
    import torch

    import fdk_b200 as F
    from fdk_b200 import phantom as P

    p = F.config(args.config)
    batch, reps = args.bp_batch, args.reps
    only = set(args.variants.split(",")) if args.variants else None
    keep = lambda name: only is None or name in only  # noqa: E731
    nu, nv = p.nu, p.nv
    s = float(1.0 / (p.SOD * p.SOD * p.AngularAndrampFactor))
    views = torch.empty((batch, nv, nu), dtype=torch.float32, device="cuda")
    P.project(p, P.phantom_for(p, 4, 20), 0, batch, views.data_ptr())
    out = torch.empty((batch, nu, nv, 2), dtype=torch.float16, device="cuda")
    frame = nu * nv
    W = int(F.lib().fdk_filter_length(nu))
    res = {"kernel": "filter", "workload": f"{args.config}: {batch} views of {nu}x{nv} per batch, W = {W}",
           "variants": {}}
    if keep("fft"):
        eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32, pad_edge=4)
        ms = timed(lambda: eng.run_device(views.data_ptr(), out.data_ptr(), batch, F.LAYOUT_MIRROR, F.DTYPE_F16, s),
                   reps)
        res["variants"]["fft"] = {"ms": ms, "hbm_gbs": batch * frame * 8 / (ms * 1e-3) / 1e9}
    flops = 2.0 * batch * nv * nu * nu
    for dt, split in (("f16", False), ("bf16", False), ("f16", True), ("bf16", True)):
        name = f"toeplitz_{dt}{'_split' if split else ''}"
        if not keep(name):
            continue
        tf = F.ToeplitzFilter(p.cos_sigma, p.fft_kernel_real, 4, dt, in_scale=s, split=split)
        ms = timed(lambda: tf.run_device(views.data_ptr(), out.data_ptr(), batch, F.LAYOUT_MIRROR, 1.0), reps)
        tf.check()
        res["variants"][name] = {"ms": ms, "tflops": (3 if split else 1) * flops / (ms * 1e-3) / 1e12}
        tf.close()
    print(json.dumps(res), flush=True)


def kernel_rtk(args) -> None:
    """The RTK drop-in on device-resident views (fdk_rtk_backproject_device): a 512^3 FP32 volume
    from 32 views of 512^2 (c2 geometry, seeded 20-ellipsoid phantom projected on the GPU), circular
    matrices and tilted ones (m[2] += 0.02 std(m[0]), m[10] += 1e-3, so u and w depend on z); the
    staged kernel ("tma") and the L1-gather kernel ("l1", FDK_RTK_KERNEL=l1)."""
    import torch

    import fdk_b200 as F
    from fdk_b200.backprojection import rtk_backproject_device, rtk_sync
    from fdk_b200.phantom import phantom_for, project

    n, W, nviews = 512, 512, 32
    p = F.config("c2")
    p.nx = p.ny = p.nz = n
    p.nu = p.nv = W
    p.nProj = nviews
    dev = torch.empty((nviews, W, W), dtype=torch.float32, device="cuda")
    project(p, phantom_for(p, 2, 20), 0, nviews, dev.data_ptr())
    vin = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    vout = torch.empty_like(vin)
    size = (W, W, nviews), (n, n, n)
    for geo in ("circular", "tilted"):
        mats = p.proj_matrices(np.float64)
        if geo == "tilted":
            mats[:, 2] += 0.02 * mats[:, 0].std()
            mats[:, 10] += 1e-3
        mats = mats.astype(np.float32)
        for kern in (args.variants.split(",") if args.variants else ["tma", "l1"]):
            if kern == "l1":
                os.environ["FDK_RTK_KERNEL"] = "l1"
            else:
                os.environ.pop("FDK_RTK_KERNEL", None)
            run = lambda: rtk_backproject_device(*size, mats, vin.data_ptr(), vout.data_ptr(), dev.data_ptr())  # noqa
            ms = timed(run, args.reps)
            rtk_sync()
            print(json.dumps({"kernel": "rtk", "geometry": geo, "variant": kern, "ms": ms,
                              "gups": n ** 3 * nviews / (ms * 1e-3) / 1e9}), flush=True)


def kernel_learned(args) -> None:
    """The learned-filter training step on the C5 geometry (256^3 volume, 90 views of 256^2): one
    noisy scan, then --reps forward + loss + gradient passes (network forward, backprojection,
    volume MSE, backprojection adjoint, network backward); about 0.3 GB on the device."""
    import torch

    from fdk_b200 import learned as Lr

    pl = Lr.Pipeline()
    p = pl.p
    x = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device=pl.dev)
    pl.scan(1000, x)
    w = torch.from_numpy(Lr.init_params()).to(pl.dev)
    w[-(32 * 9 + 1):] = 0.01
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.reps):
        pl.truth_of(1000)
        pl.reconstruct(w, x)
        e = pl.mse(True)
        pl.gradient(w, x)
    torch.cuda.synchronize()
    print(json.dumps({"kernel": "learned", "steps": args.reps,
                      "ms_per_step": 1e3 * (time.perf_counter() - t0) / args.reps, "mse": e}), flush=True)


def pairs_views(param, precision: str) -> bool:
    """Whether the reconstructor pairs views into quarter-turn quadruples for this precision by
    default (fdk_recon_bp_kernel): FP32 (MIXED with FDK_BP_SYM=1) on a square grid from a scan of
    N % 4 == 0 views; the library's own checks decide in the end."""
    sym = os.environ.get("FDK_BP_SYM", "")
    on = (precision == "fp32" and sym != "0") or (precision == "mixed" and sym == "1")
    return on and param.nx == param.ny and param.nProj % 4 == 0


def main():
    global BATCH, READ_ORDER
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=128)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp32_exact"])
    ap.add_argument("--config", default=None, help="c1..c5 (default c3; kernel benches: their own)")
    ap.add_argument("--bp-batch", type=int, default=None, help="views per backprojection batch")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP32, accuracy and reference-GPU legs")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-full", action="store_true", help="time the reference CPU FDK on the whole workload")
    ap.add_argument("--kernel", choices=["bp", "filter", "rtk", "learned"], default=None)
    ap.add_argument("--batches", type=int, default=3, help="--kernel bp: batches")
    ap.add_argument("--reps", type=int, default=3, help="--kernel filter/rtk/learned: timed repetitions")
    ap.add_argument("--variants", default="", help="--kernel filter/rtk: comma-separated variants")
    ap.add_argument("--read-order", choices=["auto", "quarter", "sequential"], default="auto",
                    help="views per step: 8 from each quarter of the scan, or 32 consecutive (auto: quarter "
                         "where the reconstructor pairs views)")
    args = ap.parse_args()
    if args.kernel:
        defaults = {"bp": ("c2", 128), "filter": ("c4", 128), "rtk": ("c2", 32), "learned": ("c5", 90)}
        args.config = args.config or defaults[args.kernel][0]
        args.bp_batch = args.bp_batch or defaults[args.kernel][1]
        {"bp": kernel_bp, "filter": kernel_filter, "rtk": kernel_rtk, "learned": kernel_learned}[args.kernel](args)
        return
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    BATCH = args.bp_batch or BATCH
    from fdk_b200.geometry import config

    param = config(args.config or "c3")
    READ_ORDER = args.read_order if args.read_order != "auto" else (
        "quarter" if pairs_views(param, args.precision) else "sequential")
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, param, rank)
    else:
        run_ours(args, param, rank, world, local)


if __name__ == "__main__":
    main()
