"""The C ABI library: loads without a GPU, exports every symbol include/fdk.h declares, and
reports errors through status codes (never crashes or throws) -- no compute calls here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "fdk.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdk_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(L, name), name


def test_abi_version_and_device_count():
    assert F.lib().fdk_abi_version() == 1
    assert F.device_count() >= 0


def test_invalid_arguments_return_status():
    L = F.lib()
    h = C.c_void_p()
    top = F.BoxT(0, 0, 0, 8, 8, 4)
    bot = F.BoxT(0, 0, 3, 8, 8, 4)  # violates the mirror rule
    rc = L.fdk_bp_create(C.byref(h), 8, 8, 4, 8, 8, 8, C.byref(top), C.byref(bot), 0, 0)
    assert rc == -1 and b"nz - 1" in L.fdk_last_error()
    rc = L.fdk_bp_create(C.byref(h), 8, 8, 500, 8, 8, 8, C.byref(top), C.byref(top), 0, 0)
    assert rc == -1
    out = np.zeros(4, np.float64)
    assert L.fdk_filter_design(9, 64, 1, out.ctypes.data, 4) == -1
    assert L.fdk_filter_design(5, 64, 1, out.ctypes.data, 4) == -1  # capacity < W
    g = F.config("c1").to_c()
    g.sod = 2000.0  # SOD > SID
    assert L.fdk_cos_table(C.byref(g), out.ctypes.data) == -1


@pytest.mark.skipif(F.device_count() > 0, reason="checks the no-GPU error path")
def test_no_device_is_an_error_not_a_crash():
    L = F.lib()
    h = C.c_void_p()
    top = F.BoxT(0, 0, 0, 8, 8, 4)
    bot = F.BoxT(0, 0, 4, 8, 8, 4)
    rc = L.fdk_bp_create(C.byref(h), 8, 8, 4, 8, 8, 8, C.byref(top), C.byref(bot), 0, 0)
    assert rc in (-2, -6) and not h.value
    with pytest.raises(F.FdkError):
        F.Reconstructor(F.config("c1"), "mixed")
