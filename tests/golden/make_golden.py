"""Writes tests/golden/ref_cpu.npz: outputs of the reference's own CPU code, compiled from its
sources by oracle/build_ref.sh (oracle/_ref/libref_cpu.so), on small seeded inputs.

    python tests/golden/make_golden.py        (needs oracle/_ref/libref_cpu.so)

The reference ships no golden vectors, known-answer tests or fixtures for this path (its Test/
folder is an empty googletest demo, its data folders are external), so these are made here from
its code and committed, so that tests/test_golden.py pins the oracle without the reference tree:

* filter(): the frequency response of all six windows (common/type.h:4427-4475) at nu = 60, 64, 256
  (W = 128, 128, 512), and hann at nu = 1536 (W = 4096);
* Parameter::init's cosine table and CalculateProjMat's matrices (type.h:4756-4833, 4898-4944) of a
  32^3 geometry with detector offsets and a volume position angle;
* the Bourke row filter filterImageRow (type.h:4169-4239) of 7 seeded rows of 60;
* 3dct's CPU FDK BackProjection<float> (3dct/3dct.cpp:3-241) of a 32^3 volume from 16 views of 32^2
  of one ellipsoid (the projections are stored too);
* 3dct's ray marcher ForwardProjection<float> (3dct/3dct.cpp:430-573) of a seeded 48^3
  random-ellipsoid volume, 6 views of 56 x 40.

The inputs are deterministic: seeded generators and the oracle's FP64 analytic projector."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

WINDOWS = ["none", "ram-lak", "shepp-logan", "cosine", "hamming", "hann"]
ELLIPSOID = np.array([[12.0, -20.0, 10.0, 60.0, 40.0, 50.0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 1.0]])


def small(n=32, views=16):
    from fdk_b200 import config

    p = config("c1")
    p.nx = p.ny = p.nz = n
    p.dx = p.dy = p.dz = 256.0 / n
    p.nu = p.nv = n
    p.du = p.dv = 384.0 / n
    p.nProj = views
    return p


def cos_geometry():
    p = small(32, views=24)
    p.offset_nu, p.offset_nv = 1.25, -0.5
    p.volume_postion_angle = 0.3
    return p


def fproj_geometry():
    from tests.helpers import small_param

    return small_param(48, 56, 40, 6)


def fproj_volume(p):
    from fdk_b200.phantom import phantom_for

    return O.ellipsoid_volume(phantom_for(p, 4, 12), p)


def fdk_projections(p):
    return np.stack([O.ellipsoid_projection(ELLIPSOID, p, a) for a in O.view_angles(p)]).astype(np.float32)


def rows_input():
    return np.random.default_rng(1).standard_normal((7, 60)).astype(np.float32)


def main() -> None:
    R = O.RefCPU()
    out = {}
    for nu in (60, 64, 256):
        p = small()
        p.nu = nu
        for w in WINDOWS:
            out[f"H_{w}_{nu}"] = R.parameter(p, w)["H"]
    p = small()
    p.nu = 1536
    out["H_hann_1536"] = R.parameter(p, "hann")["H"]
    g = cos_geometry()
    par = R.parameter(g)
    out["cos"], out["mats"] = par["cos"], par["mats"]
    src = rows_input()
    out["rows_H"] = O.filter_design("hann", src.shape[1])
    out["rows_out"] = R.filter_rows(out["rows_H"], src)
    p = small(32, views=16)
    proj = fdk_projections(p)
    vol = np.zeros((p.nz, p.ny, p.nx), np.float32)
    R.cpu_fdk(p, proj, 0, vol)
    out["fdk_proj"], out["fdk_vol"] = proj, vol
    q = fproj_geometry()
    v = fproj_volume(q)
    out["fproj"] = np.stack([R.forward_projection(v, q, i) for i in range(q.nProj)])
    path = os.path.join(HERE, "ref_cpu.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
