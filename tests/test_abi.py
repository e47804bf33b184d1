"""The C ABI: library loads, exports every declared symbol, host-side checks
behave without a GPU (no compute call is made here)."""
import ctypes
import os
import re

import numpy as np

from sqcalc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(sqn_[a-z0-9_]+)\s*\(", text))
    return names


def test_exports_every_declared_symbol(sqn_lib):
    names = declared_symbols()
    assert names, "no declarations found"
    for n in sorted(names):
        assert hasattr(sqn_lib, n), n
    assert set(_lib.EXPORTS) <= names


def test_abi_version_and_errors(sqn_lib):
    assert sqn_lib.sqn_abi_version() == _lib.ABI_VERSION
    assert _lib.error_string(0) == "ok"
    assert "mode limit" in _lib.error_string(42)
    assert "unknown" in _lib.error_string(12345)


def test_default_desc_matches_sqcalc_defaults(sqn_lib):
    d = _lib.SqnDesc()
    sqn_lib.sqn_default_desc(ctypes.byref(d))
    # src/sqc_options.f90:51-140 and src/sqc_structure_factor.f90:74-86
    assert (d.qmin, d.qmax, d.nq, d.eps) == (0.0, 20.0, 500, 1e-9)
    assert d.norm == _lib.NORM_MEAN and d.partials == 1 and d.weight == _lib.WEIGHT_UNIT
    assert d.precision == _lib.PREC_DOUBLE and d.abi_version == _lib.ABI_VERSION


def test_bad_arguments_are_status_codes_not_crashes(sqn_lib):
    h = ctypes.c_void_p()
    assert sqn_lib.sqn_plan_create(None, ctypes.byref(h)) == 21
    d = _lib.SqnDesc()
    sqn_lib.sqn_default_desc(ctypes.byref(d))
    d.abi_version = 999
    assert sqn_lib.sqn_plan_create(ctypes.byref(d), ctypes.byref(h)) == 40
    assert not h.value
    assert sqn_lib.sqn_sync(None) == 16
    assert sqn_lib.sqn_plan_destroy(None) == 16
    assert sqn_lib.sqn_launch_count(None) == -1


def test_plan_without_gpu_reports_no_device(sqn_lib):
    import torch
    if torch.cuda.is_available():
        return
    types = np.ones(10, dtype=np.int32)
    d = _lib.SqnDesc()
    sqn_lib.sqn_default_desc(ctypes.byref(d))
    d.natoms = 10
    d.ntypes = 1
    d.type_id = types.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    h = ctypes.c_void_p()
    assert sqn_lib.sqn_plan_create(ctypes.byref(d), ctypes.byref(h)) == 41
    assert not h.value
