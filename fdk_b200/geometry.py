"""Parameter: the reference's FDK geometry core (common/type.h:4627-4895) over the C ABI.

Field names follow the reference (``SID`` is source-to-detector, ``SOD`` source-to-axis,
``volume_postion_angle`` keeps its spelling); all tables are computed by libfdk_b200 in FP64.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import FILTERS, Geometry, check, lib


@dataclass
class Parameter:
    nx: int = 512
    ny: int = 512
    nz: int = 512
    dx: float = 0.157
    dy: float = 0.157
    dz: float = 0.146
    nu: int = 608
    nv: int = 616
    du: float = 0.2
    dv: float = 0.2
    offset_nu: float = 0.0
    offset_nv: float = 0.0
    SID: float = 700.0
    SOD: float = 468.0
    direction: int = -1
    scan_angle: float = 360.0
    nProj: int = 512
    volume_postion_angle: float = -np.pi * 48.8671875 / 180.0
    str_filter: str = "shepp-logan"

    # ------------------------------------------------------------------ C struct
    def to_c(self) -> Geometry:
        g = Geometry()
        g.nx, g.ny, g.nz = self.nx, self.ny, self.nz
        g.dx, g.dy, g.dz = self.dx, self.dy, self.dz
        g.nu, g.nv = self.nu, self.nv
        g.du, g.dv = self.du, self.dv
        g.offset_nu, g.offset_nv = self.offset_nu, self.offset_nv
        g.sid, g.sod = self.SID, self.SOD
        g.direction, g.scan_angle, g.n_proj = self.direction, self.scan_angle, self.nProj
        g.volume_position_angle = self.volume_postion_angle
        g.filter_type = FILTERS[self.str_filter]
        return g

    # ------------------------------------------------------------------ tables (init())
    @property
    def filter_length(self) -> int:
        """nextpow2(nu) (common/type.h:4418-4425)."""
        return int(lib().fdk_filter_length(self.nu))

    @property
    def fft_kernel_real(self) -> np.ndarray:
        """filter(str_filter, nu, 1) (common/type.h:4427-4475), FP64."""
        W = self.filter_length
        out = np.zeros(W, np.float64)
        check(lib().fdk_filter_design(FILTERS[self.str_filter], self.nu, 1, out.ctypes.data, W))
        return out

    @property
    def fft_kernel_real_f32(self) -> np.ndarray:
        return self.fft_kernel_real.astype(np.float32)

    @property
    def AngularAndrampFactor(self) -> float:
        v = C.c_double(0)
        check(lib().fdk_angular_ramp_factor(C.byref(self.to_c()), C.byref(v)))
        return v.value

    @property
    def cos_sigma(self) -> np.ndarray:
        """cos_image_table.cos_sigma, nv rows x nu (common/type.h:4756-4783)."""
        out = np.zeros((self.nv, self.nu), np.float32)
        check(lib().fdk_cos_table(C.byref(self.to_c()), out.ctypes.data))
        return out

    @property
    def csc_sigma(self) -> np.ndarray:
        """cos_image_table.csc_sigma = 1 / cos_sigma, nv rows x nu (common/type.h:4760, 4784)."""
        out = np.zeros((self.nv, self.nu), np.float32)
        check(lib().fdk_csc_table(C.byref(self.to_c()), out.ctypes.data))
        return out

    @property
    def angles(self) -> np.ndarray:
        """direction * vec_deg / 180 * pi + volume_postion_angle per view (radians)."""
        out = np.zeros(self.nProj, np.float64)
        check(lib().fdk_view_angles(C.byref(self.to_c()), out.ctypes.data))
        return out

    def proj_matrices(self, dtype=np.float32) -> np.ndarray:
        """vec_rot_mat_ijk3x4 as (nProj, 12) (CalculateProjMat, common/type.h:4898-4944)."""
        out64 = np.zeros((self.nProj, 12), np.float64)
        out32 = np.zeros((self.nProj, 12), np.float32)
        check(lib().fdk_projection_matrices(C.byref(self.to_c()), out64.ctypes.data, out32.ctypes.data))
        return out64 if dtype == np.float64 else out32

    @property
    def vec_rot_mat_ijk3x4(self) -> np.ndarray:
        return self.proj_matrices(np.float32).reshape(-1)


def default_parameter() -> Parameter:
    """Parameter::Parameter() defaults, read back from the library (common/type.h:4628-4662)."""
    g = Geometry()
    lib().fdk_geometry_default(C.byref(g))
    inv = {v: k for k, v in FILTERS.items()}
    return Parameter(nx=g.nx, ny=g.ny, nz=g.nz, dx=g.dx, dy=g.dy, dz=g.dz, nu=g.nu, nv=g.nv, du=g.du, dv=g.dv,
                     offset_nu=g.offset_nu, offset_nv=g.offset_nv, SID=g.sid, SOD=g.sod, direction=g.direction,
                     scan_angle=g.scan_angle, nProj=g.n_proj, volume_postion_angle=g.volume_position_angle,
                     str_filter=inv[g.filter_type])


def config(name: str) -> Parameter:
    """The benchmark geometries (SOD 1000 mm, SID 1500 mm, Hann window, views over 360 deg,
    volume_postion_angle 0).  c1: 256^3 1 mm / 256^2 1.5 mm, 256 views; c2: 512^3, 512 views;
    c3: 2048^3, 4096 views of 2048^2; c4: 1024^3, 1024 views of 1536 x 1024; c5: 256^3, 90 views.
    c2-c4 keep c1's field of view (256 mm volume, 384 mm detector width) with scaled pitch."""
    base = dict(SOD=1000.0, SID=1500.0, direction=-1, scan_angle=360.0, volume_postion_angle=0.0,
                str_filter="hann", offset_nu=0.0, offset_nv=0.0)
    table = {
        "c1": dict(nx=256, ny=256, nz=256, dx=1.0, dy=1.0, dz=1.0, nu=256, nv=256, du=1.5, dv=1.5, nProj=256),
        "c2": dict(nx=512, ny=512, nz=512, dx=0.5, dy=0.5, dz=0.5, nu=512, nv=512, du=0.75, dv=0.75, nProj=512),
        "c3": dict(nx=2048, ny=2048, nz=2048, dx=0.125, dy=0.125, dz=0.125, nu=2048, nv=2048, du=0.1875,
                   dv=0.1875, nProj=4096),
        "c4": dict(nx=1024, ny=1024, nz=1024, dx=0.25, dy=0.25, dz=0.25, nu=1536, nv=1024, du=0.25, dv=0.25,
                   nProj=1024),
        "c5": dict(nx=256, ny=256, nz=256, dx=1.0, dy=1.0, dz=1.0, nu=256, nv=256, du=1.5, dv=1.5, nProj=90),
    }
    return Parameter(**base, **table[name])
