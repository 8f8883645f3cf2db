"""The C++ drop-in header (include/fdk.hpp) builds against the C ABI and, on a GPU, runs the
reference pipeline's call sequence with results equal to the Python binding's."""
import os
import subprocess

import numpy as np
import pytest

from fdk_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "drop_in.cpp")


def build_drop_in(tmp_path) -> str:
    exe = str(tmp_path / "drop_in")
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                           "-L", libdir, "-l:libfdk_b200.so", f"-Wl,-rpath,{libdir}"])
    return exe


def test_cpp_header_compiles_and_links(tmp_path):
    exe = build_drop_in(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_cpp_drop_in_pipeline(tmp_path, precision):
    import fdk_b200 as F
    from tests.helpers import knife_edge_mask, phantom_views, rel_l2, small_param

    exe = build_drop_in(tmp_path)
    n, views = 32, 40
    p = small_param(n, 40, 40, views)
    _, proj = phantom_views(p, seed=9)
    vin, vout = tmp_path / "views.f32", tmp_path / "vol.f32"
    proj.astype(np.float32).tofile(vin)
    r = subprocess.run([exe, str(vin), str(vout), str(n), "40", "40", str(views), str(precision)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "nBpCount=40" in r.stdout
    got = np.fromfile(vout, np.float32).reshape(n, n, n)
    # the same sequence through the Python binding
    eng = F.FilterEngine(p.cos_sigma, p.fft_kernel_real_f32)
    bp = F.BackProjectionFDK(p.nv, p.nu, 32, n, n, n, F.BoxT(0, 0, 0, n, n, n // 2), F.BoxT(0, 0, n // 2, n, n, n // 2),
                             ["fp32_exact", "fp32", "mixed"][precision])
    mats = p.proj_matrices()
    filt = np.zeros((views, p.nu, p.nv), np.float32)
    for s in range(views):
        eng.Filtering(proj[s].copy(), filt[s], True)
    for i in range(0, views, 32):
        bp.BP(1, filt[i:i + 32], p.nv, p.nu, mats[i:i + 32], min(32, views - i))
    want = bp.GetVolumeData()
    if precision == 0:
        assert np.array_equal(got, want)
    else:
        m = knife_edge_mask(p, [0, 0, 0, n, n, n // 2], n // 2)
        assert rel_l2(got[m], want[m]) <= 1e-6
