"""On-disk formats (projection folders, .vol volumes, per-slice files) and the csc_sigma table.
Host code only; the files are cross-checked against numpy's own raw writer/reader."""
import os

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200 import formats as FM
from fdk_b200._lib import FdkError
from tests.helpers import small_param


def test_proj_path_follows_get_proj_path():
    # GetProjPath: folder + "img%04d.raw" % (index * step) (common/type.h:4847-4851)
    assert FM.proj_path("/data/p/", 7) == "/data/p/img0007.raw"
    assert FM.proj_path("/data/p", 7, step=3) == "/data/p/img0021.raw"
    assert FM.proj_path("rel/", 12345, step=1, start=2) == "rel/img12347.raw"


def test_projection_folder_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    views = rng.standard_normal((5, 6, 7)).astype(np.float32)  # (n, nv, nu)
    folder = str(tmp_path / "proj")
    FM.save_proj_folder(folder, views, first=0, step=2)
    names = sorted(os.listdir(folder))
    assert names == [f"img{2 * i:04d}.raw" for i in range(5)]
    # raw little-endian FP32, u fastest: numpy reads each file back as one view
    for i in range(5):
        np.testing.assert_array_equal(np.fromfile(os.path.join(folder, names[i]), "<f4").reshape(6, 7), views[i])
    got = FM.load_proj_folder(folder, nu=7, nv=6, count=3, first=1, step=2, threads=3)
    np.testing.assert_array_equal(got, views[1:4])


def test_loader_reads_files_written_by_numpy(tmp_path):
    rng = np.random.default_rng(1)
    views = rng.standard_normal((4, 3, 5)).astype(np.float32)
    for i, v in enumerate(views):
        v.astype("<f4").tofile(str(tmp_path / f"img{i + 10:04d}.raw"))
    got = FM.load_proj_folder(str(tmp_path), nu=5, nv=3, count=4, start=10)
    np.testing.assert_array_equal(got, views)


def test_loader_refuses_wrong_or_missing_files(tmp_path):
    views = np.zeros((3, 4, 4), np.float32)
    FM.save_proj_folder(str(tmp_path), views)
    np.zeros(15, np.float32).tofile(str(tmp_path / "img0001.raw"))  # one value short
    with pytest.raises(FdkError) as e:
        FM.load_proj_folder(str(tmp_path), 4, 4, 3)
    assert e.value.code == -8 and "img0001.raw" in str(e.value) and "wrong size" in str(e.value)
    with pytest.raises(FdkError) as e:
        FM.load_proj_folder(str(tmp_path), 4, 4, 1, first=5)
    assert e.value.code == -8 and "img0005.raw" in str(e.value) and "missing" in str(e.value)


def test_vol_round_trip_and_header(tmp_path):
    rng = np.random.default_rng(2)
    vol = rng.standard_normal((3, 4, 5)).astype(np.float32)  # [z][y][x]
    path = str(tmp_path / "sub" / "v.vol")
    FM.save_volume(path, vol)
    raw = open(path, "rb").read()
    assert np.frombuffer(raw[:12], "<i4").tolist() == [5, 4, 3]
    np.testing.assert_array_equal(np.frombuffer(raw[12:], "<f4").reshape(3, 4, 5), vol)
    np.testing.assert_array_equal(FM.load_volume(path), vol)
    with open(path, "ab") as f:
        f.write(b"\0\0\0\0")
    with pytest.raises(FdkError) as e:
        FM.load_volume(path)
    assert e.value.code == -8


def test_volume_slices(tmp_path):
    vol = np.arange(2 * 3 * 4, dtype=np.float32).reshape(2, 3, 4)
    FM.save_volume_slices(str(tmp_path / "slices"), vol, z0=40, threads=2)
    assert sorted(os.listdir(tmp_path / "slices")) == ["000040.raw", "000041.raw"]
    np.testing.assert_array_equal(np.fromfile(str(tmp_path / "slices" / "000041.raw"), "<f4").reshape(3, 4), vol[1])


def test_csc_table_is_reciprocal_of_cos_table():
    p = small_param(32, 40, 24, 8)
    cos = p.cos_sigma
    csc = p.csc_sigma
    np.testing.assert_array_equal(csc, (1.0 / cos.astype(np.float64)).astype(np.float32))
    p5 = F.config("c5")
    np.testing.assert_allclose(p5.csc_sigma * p5.cos_sigma, 1.0, rtol=1e-6)
