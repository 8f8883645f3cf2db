"""Product geometry (libfdk_b200, FP64) against the oracle and the reference's own code."""
import os

import numpy as np
import pytest

import fdk_b200 as F
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "libref_cpu.so")),
                               reason="reference CPU build absent")


@pytest.mark.parametrize("cfg", ["c1", "c2", "c4", "c5"])
def test_filter_length(cfg):
    p = F.config(cfg)
    assert p.filter_length == O.nextpow2(p.nu)
    assert F.lib().fdk_filter_length(256) == 512 and F.lib().fdk_filter_length(1536) == 2048


@pytest.mark.parametrize("ftype", list(O.FILTERS))
def test_filter_design_exact(ftype):
    p = F.config("c4")
    p.str_filter = ftype
    assert np.array_equal(p.fft_kernel_real, O.filter_design(ftype, p.nu))


@needs_ref
@pytest.mark.parametrize("cfg", ["c1", "c4"])
def test_cos_table_within_one_ulp_of_reference(cfg):
    p = F.config(cfg)
    p.nProj = 8
    ref = O.RefCPU().parameter(p)["cos"]
    got = p.cos_sigma
    assert np.abs(got.view(np.int32) - ref.view(np.int32)).max() <= 1
    assert p.AngularAndrampFactor == O.RefCPU().parameter(p)["aaf"]


@needs_ref
@pytest.mark.parametrize("vpa", [0.0, -np.pi * 48.8671875 / 180.0])
def test_projection_matrices(vpa):
    p = F.config("c2")
    p.nProj = 64
    p.volume_postion_angle = vpa
    m64 = p.proj_matrices(np.float64)
    assert np.abs(m64 - O.proj_matrices(p)).max() <= 1e-13 * np.abs(m64).max()
    ref = O.RefCPU().parameter(p)["mats"]
    assert np.abs(m64 - ref).max() <= 4e-7 * np.abs(m64).max()
    assert np.all(m64[:, 2] == 0) and np.all(m64[:, 10] == 0)


def test_matrix_maps_centre_to_detector_centre():
    p = F.config("c1")
    m = p.proj_matrices(np.float64)
    c = np.array([(p.nx - 1) / 2, (p.ny - 1) / 2, (p.nz - 1) / 2, 1.0])
    for row in m:
        M = row.reshape(3, 4)
        uw, vw, w = M @ c
        assert abs(w - p.SOD) < 1e-9
        assert abs(uw / w - (p.nu - 1) / 2) < 1e-9 and abs(vw / w - (p.nv - 1) / 2) < 1e-9


def test_mirror_symmetry_of_matrices():
    """v(nz-1-z) = nv-1-v(z): the identity the slab-pair kernels rely on."""
    p = F.config("c2")
    p.nProj = 16
    rng = np.random.default_rng(0)
    for row in p.proj_matrices(np.float64):
        M = row.reshape(3, 4)
        for _ in range(20):
            x, y, z = rng.uniform(0, p.nx - 1), rng.uniform(0, p.ny - 1), rng.uniform(0, p.nz - 1)
            a = M @ [x, y, z, 1]
            b = M @ [x, y, p.nz - 1 - z, 1]
            assert abs(a[0] / a[2] - b[0] / b[2]) < 1e-9
            assert abs(a[1] / a[2] + b[1] / b[2] - (p.nv - 1)) < 1e-9


def test_default_parameter_matches_reference_defaults():
    d = F.default_parameter()
    assert (d.nx, d.nu, d.nv, d.nProj, d.str_filter) == (512, 608, 616, 512, "shepp-logan")
    assert d.SOD == 468 and d.SID == 700.0 and d.direction == -1
    assert abs(d.volume_postion_angle - (-np.pi * 48.8671875 / 180.0)) < 1e-15


def test_angles():
    p = F.config("c5")
    a = p.angles
    assert a.shape == (90,)
    assert np.allclose(a, O.view_angles(p))
