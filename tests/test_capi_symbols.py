"""The C-ABI library loads and exports every entry point include/fcb200.h declares.

No compute call is made here (this file runs without a GPU).
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\bint\s+(fcb200_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["fcb200_third_order_lj", "fcb200_mass_weight3", "fcb200_mcc3", "fcb200_mcc3_blocked",
                 "fcb200_snapshot_lj", "fcb200_last_error", "fcb200_create", "fcb200_destroy"]:
        assert must in names


def test_library_exports_every_declared_symbol(fcb):
    from fcb200 import _lib
    L = _lib.lib()
    for name in declared_symbols():
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature in fcb200/_lib.py"


def test_version_and_last_error(fcb):
    from fcb200 import _lib
    assert _lib.lib().fcb200_version() >= 100
    code, msg = _lib.last_error()
    assert isinstance(msg, str)


def test_create_without_gpu_reports_status(fcb):
    """On a machine without a CUDA device, create fails with a status, not a crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fcb200 import _lib
    h = ctypes.c_void_p()
    st = _lib.lib().fcb200_create(ctypes.byref(h), 0)
    assert st == _lib.FCB_ERR_UNSUPPORTED
    assert h.value is None
    assert "no CUDA device" in _lib.last_error()[1]


def test_null_handle_is_an_argument_error(fcb):
    from fcb200 import _lib
    L = _lib.lib()
    assert L.fcb200_third_order_lj(None, None, 0, None, 0, 0, 0, 0, None, None, None, 0, None) == _lib.FCB_ERR_ARG
    assert L.fcb200_mcc3(None, None, None, 0, 0, 0, 0, 0, 0, 0, 0, None, None) == _lib.FCB_ERR_ARG
    assert L.fcb200_destroy(None) == _lib.FCB_OK
    assert L.fcb200_set_wait_limit(None, 1) == _lib.FCB_ERR_ARG
