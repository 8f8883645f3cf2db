"""The benchmark geometries at their full sizes on the GPU, and the paths that only show at size.

* C1 (256^3 from 256 views of 256^2) and C2 (512^3 from 512 views of 512^2), all three
  precisions: FP32_EXACT bit for bit against the reference's own cudaFdkBP (compiled for sm_100a)
  on the same filtered views; every precision against the FP64 oracle (filter + backprojection
  in double) at 1e5 seeded voxels and every voxel of the central x, y and z slices; the
  reference's CPU FDK (3dct) against the same FP64 oracle (with its 3-sample pad) and against
  the GPU result.  Errors are reported over all sampled voxels and without the knife-edge
  voxels (projected within 1e-3 px of a detector border in some view, where the reference's
  bounds rule is discontinuous).
* A 512^3 slab pair (C2 geometry): MIXED against FP64 and FP32 (staged) against the reference
  arithmetic (FP32_EXACT).
* The multi-GPU path on one GPU: the slab-pair reconstructors of a 4-way DivVolume
  (cuFDK/mpiFDK.h:116-149) against the single-GPU volume.
* The staged kernel's bounded device wait, made to run out on purpose (a pipeline stage its
  producer never fills; no GPU fault): the host gets FDK_ERR_DEVICE_CHECK, and the same handle
  then reconstructs correctly after a reset.

C1's modified Shepp-Logan phantom comes from an external script that is not available here, so
both configs use the seeded random-ellipsoid phantom instead (C1: 10 ellipsoids, C2: 20).
"""
import os

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200.phantom import phantom_for, project
from fdk_b200.shard import div_volume
from oracle import oracle as O
from tests.helpers import rel_l2, small_param

pytestmark = pytest.mark.gpu

REF_GPU = os.path.exists(os.path.join(O.REF_DIR, "libref_gpu_bp.so"))
REF_CPU = os.path.exists(os.path.join(O.REF_DIR, "libref_cpu.so"))


def _views(p, seed, n_ell):
    import torch

    ell = phantom_for(p, seed, n_ell)
    dev = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device="cuda")
    project(p, ell, 0, p.nProj, dev.data_ptr())
    torch.cuda.synchronize()
    return dev


def _recon(p, precision, dev, slab=None, batch=None):
    """Reconstructor fed from device views; the staged precisions read 8 consecutive views from
    each quarter of the scan in turn, so batches pair views with their quarter-turn partners."""
    r = F.Reconstructor(p, precision, batch=batch or (32 if precision == "fp32_exact" else 256), slab=slab)
    if precision == "fp32_exact" or p.nProj % 32:
        for c in range(0, p.nProj, 32):
            r.push_device(dev[c:].data_ptr(), c, min(32, p.nProj - c))
    else:
        q = p.nProj // 4
        for b in range(0, q, 8):
            for k in range(4):
                r.push_device(dev[b + k * q:].data_ptr(), b + k * q, 8)
    return r


def _err(got, want, mask):
    e = {"all": rel_l2(got, want)}
    e["masked"] = rel_l2(got[~mask], want[~mask]) if mask.any() else e["all"]
    return e


def _full_size_check(cfg, seed, n_ell, cpu_slab):
    """All precisions of one benchmark config at full size; returns the measured errors."""
    import torch

    p = F.config(cfg)
    n = p.nx
    dev = _views(p, seed, n_ell)
    host = dev.cpu().numpy()
    vox = O.sample_voxels(n, n, n, 100000, seed)
    got = {}
    for prec in ("fp32_exact", "fp32", "mixed"):
        r = _recon(p, prec, dev)
        got[prec] = r.sample(vox)
        r.close()
    S4 = O.SampledFDK(p, vox, pad_n=4)  # the reconstructor's filter pad (the IPP plugin)
    for c in range(0, p.nProj, 64):
        S4.add(host[c:c + 64], c)
    edge = S4.edge.astype(bool)
    errs = {prec: _err(got[prec], S4.values, edge) for prec in got}
    errs["fp32_vs_exact"] = _err(got["fp32"], got["fp32_exact"], edge)
    print(cfg, errs)
    assert errs["mixed"]["all"] <= 1e-3 and errs["mixed"]["masked"] <= 1e-3
    assert errs["fp32"]["masked"] <= 1e-5 and errs["fp32_exact"]["masked"] <= 1e-5
    assert errs["fp32_vs_exact"]["masked"] <= 1e-5

    if REF_GPU:
        # FP32_EXACT bit for bit against the reference kernel on the same filtered views (the
        # BackProjectionFDK boundary, 32 views per call), over the whole volume
        eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32, pad_edge=4)
        filt = torch.empty((p.nProj, p.nu, p.nv), dtype=torch.float32, device="cuda")
        eng.run_device(dev.data_ptr(), filt.data_ptr(), p.nProj, F.LAYOUT_TRANSPOSED, F.DTYPE_F32, 1.0)
        torch.cuda.synchronize()
        fh = filt.cpu().numpy()
        eng.close()
        del filt
        mats = p.proj_matrices()
        top, bot = [0, 0, 0, n, n, n // 2], [0, 0, n // 2, n, n, n // 2]
        bp = F.BackProjectionFDK(p.nv, p.nu, 32, n, n, n, F.BoxT(*top), F.BoxT(*bot), precision="fp32_exact")
        for c in range(0, p.nProj, 32):
            bp.BP(1, fh[c:c + 32], p.nv, p.nu, mats[c:c + 32], 32)
        ours = bp.GetVolumeData()
        bp.close()
        ref = O.RefGPU().backproject([fh[c:c + 32] for c in range(0, p.nProj, 32)],
                                     [mats[c:c + 32] for c in range(0, p.nProj, 32)], n, n, n, top, bot)
        assert np.array_equal(ours, ref)

    if REF_CPU:
        # 3dct on a central z-slab (the whole volume when cpu_slab >= nz): FP32 BP after an FP64
        # Bourke filter with a 3-sample pad, scaled by AngularAndrampFactor twice (3dct.cpp:43)
        import copy

        sp = copy.copy(p)
        sp.nz = min(cpu_slab, n)
        z0 = (n - sp.nz) // 2
        cpu = np.zeros((sp.nz, n, n), np.float32)
        O.RefCPU().cpu_fdk(sp, host, 0, cpu)
        cpu /= O.angular_ramp_factor(p)
        # the detector-covered core, where the two bilinear boundary rules agree
        sel = (vox[:, 2] >= z0) & (vox[:, 2] < z0 + sp.nz)
        c = (vox[:, 0] - (n - 1) / 2) ** 2 + (vox[:, 1] - (n - 1) / 2) ** 2 < (0.35 * n) ** 2
        c &= np.abs(vox[:, 2] - (n - 1) / 2) < 0.35 * n
        sel &= c
        vs = vox[sel]
        cpu_v = cpu[vs[:, 2] - z0, vs[:, 1], vs[:, 0]]
        S3 = O.SampledFDK(p, vs, pad_n=3)  # 3dct's own pad
        for k in range(0, p.nProj, 64):
            S3.add(host[k:k + 64], k)
        e3 = {"3dct_vs_fp64": rel_l2(cpu_v, S3.values), "mixed_vs_3dct": rel_l2(got["mixed"][sel], cpu_v),
              "fp32_vs_3dct": rel_l2(got["fp32"][sel], cpu_v), "voxels": int(sel.sum())}
        print(cfg, e3)
        assert e3["3dct_vs_fp64"] <= 2e-4
        # ours filters with the IPP plugin's 4-sample pad, 3dct with 3: a small, smooth difference
        assert e3["fp32_vs_3dct"] <= 2e-3 and e3["mixed_vs_3dct"] <= 2e-3
    return errs


def test_c1_full_size_all_precisions():
    _full_size_check("c1", 1, 10, cpu_slab=256)


def test_c2_full_size_all_precisions():
    _full_size_check("c2", 2, 20, cpu_slab=64)


def test_c4_full_size_mixed_and_fp32_vs_fp64():
    """C4 (1024^3 from 1024 views of 1536 x 1024): 1.5 detector pixels per voxel, so about 1% of
    the staged kernels' (tile, view) footprints exceed their shared-memory box and are gathered
    from global memory.  MIXED and FP32 against the FP64 oracle at 1e5 seeded voxels and the
    central slices."""
    p = F.config("c4")
    n = p.nx
    dev = _views(p, 4, 30)
    host = dev.cpu().numpy()
    vox = O.sample_voxels(n, n, n, 100000, 4)
    got = {}
    for prec in ("fp32", "mixed"):
        r = _recon(p, prec, dev)
        got[prec] = r.sample(vox)
        r.close()
    del dev
    S4 = O.SampledFDK(p, vox, pad_n=4)
    for c in range(0, p.nProj, 64):
        S4.add(host[c:c + 64], c)
    edge = S4.edge.astype(bool)
    errs = {prec: _err(got[prec], S4.values, edge) for prec in got}
    print("c4", errs)
    assert errs["mixed"]["all"] <= 1e-3 and errs["mixed"]["masked"] <= 1e-3
    assert errs["fp32"]["masked"] <= 1e-5


def test_c2_slab_pair_mixed_vs_fp64_and_fp32_vs_reference_arithmetic():
    """A central 2 x 64-slice slab pair of the 512^3 volume (one rank's share)."""
    p = F.config("c2")
    dev = _views(p, 5, 20)
    slab = (192, 64)
    vols = {}
    for prec in ("fp32_exact", "fp32", "mixed"):
        r = _recon(p, prec, dev, slab=slab)
        vols[prec] = r.volume().astype(np.float64)
        r.close()
    zs = np.concatenate([np.arange(192, 256), np.arange(256, 320)])
    # FP64 oracle at every voxel of 8 of the slab's slices (4 top, 4 mirror) -- 2 M voxels
    pick = np.array([0, 21, 42, 63, 64, 85, 106, 127])
    y, x = np.meshgrid(np.arange(512), np.arange(512), indexing="ij")
    vox = np.concatenate([np.stack([x.ravel(), y.ravel(), np.full(x.size, zs[k])], 1) for k in pick]).astype(np.int32)
    S = O.SampledFDK(p, vox, pad_n=4)
    host = dev.cpu().numpy()
    for c in range(0, p.nProj, 64):
        S.add(host[c:c + 64], c)
    got = {k: v[pick].reshape(-1) for k, v in vols.items()}
    edge = S.edge.astype(bool)
    e_mixed = rel_l2(got["mixed"], S.values)
    # FP32 (staged) against the reference arithmetic, without the knife-edge voxels of the sampled
    # slices (columns whose projection touches a detector border in some view); unmasked reported
    e_fp32 = rel_l2(got["fp32"][~edge], got["fp32_exact"][~edge])
    print("slab pair: mixed vs fp64", e_mixed, "fp32 vs fp32_exact", e_fp32, "unmasked whole slab",
          rel_l2(vols["fp32"], vols["fp32_exact"]), "fp32 vs fp64", rel_l2(got["fp32"], S.values),
          "knife-edge voxels", int(edge.sum()))
    assert e_mixed <= 1e-3 and e_fp32 <= 1e-5


@pytest.mark.parametrize("precision", ["fp32_exact", "fp32", "mixed"])
def test_divvolume_slab_ranks_assemble_the_single_gpu_volume(precision):
    """Ranks 0..3 of a 4-way DivVolume (each a slab-pair reconstructor, as one GPU of the
    multi-GPU path) against the whole-volume reconstructor: FP32_EXACT bit for bit (its per-voxel
    arithmetic does not depend on the slab), the staged precisions within their rounding (their
    tiles start at other z, so v is carried from other slices)."""
    p = small_param(128, 160, 128, 64)
    dev = _views(p, 7, 12)
    whole = _recon(p, precision, dev, batch=32 if precision == "fp32_exact" else 64)
    full = whole.volume().astype(np.float64)  # [z][y][x]
    whole.close()
    for rank in range(4):
        sp = div_volume(p.nx, p.ny, p.nz, rank, 4)
        r = _recon(p, precision, dev, slab=(int(sp.top.z), int(sp.top.depth)),
                   batch=32 if precision == "fp32_exact" else 64)
        got = r.volume().astype(np.float64)
        r.close()
        want = full[sp.z_indices()]
        if precision == "fp32_exact":
            assert np.array_equal(got, want), rank
        else:
            assert rel_l2(got, want) <= (1e-6 if precision == "fp32" else 1e-4), (rank, rel_l2(got, want))


@pytest.mark.parametrize("pair", [False, True])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_device_wait_timeout_reports_and_recovers(precision, pair, monkeypatch):
    """FDK_BP_TEST_WITHHOLD makes CTA 0's producer skip its first pipeline stage; with a 1 ms
    wait limit its consumers give up, set the device error word and return, the producer drains
    its own copies (bounded) -- the host sees FDK_ERR_DEVICE_CHECK at the sync.  After a reset
    (and without the switch) the handle reconstructs as before.  Both staged kernels: the
    16 views form 4 whole quarter-turn orbits (pair) or the pairing is off (FDK_BP_SYM=0)."""
    p = small_param(64, 64, 64, 16)
    dev = _views(p, 8, 8)
    monkeypatch.setenv("FDK_BP_SYM", "1" if pair else "0")
    r = F.Reconstructor(p, precision, batch=16)
    monkeypatch.delenv("FDK_BP_SYM", raising=False)
    assert r.bp_kernel == ("quarter-turn" if pair else "staged")
    r.push_device(dev.data_ptr(), 0, 16)
    want = r.volume().copy()
    r.reset()
    monkeypatch.setenv("FDK_BP_WAIT_NS", "1000000")
    monkeypatch.setenv("FDK_BP_TEST_WITHHOLD", "1")
    r.push_device(dev.data_ptr(), 0, 16)
    with pytest.raises(F.FdkError) as e:
        r.sync()
    assert e.value.code == -7 and b"timed out on the device" in F.lib().fdk_last_error()  # FDK_ERR_DEVICE_CHECK
    monkeypatch.delenv("FDK_BP_TEST_WITHHOLD")
    monkeypatch.delenv("FDK_BP_WAIT_NS")
    r.reset()
    r.push_device(dev.data_ptr(), 0, 16)
    got = r.volume()
    r.close()
    assert np.array_equal(got, want)
