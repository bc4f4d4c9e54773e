"""The C-ABI library loads and exports every symbol include/bt_gpu.h declares
(no compute calls without a GPU)."""
import ctypes as C
import os
import re

import numpy as np

from conftest import ROOT


def _declared():
    text = open(os.path.join(ROOT, "include", "bt_gpu.h")).read()
    return sorted(set(re.findall(r"BT_API\s+[\w\s\*]+?\b(bt_\w+)\s*\(", text)))


def test_exports_every_declared_symbol(native_lib):
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(native_lib, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_ctypes_signature(native_lib):
    """The Python binding (_native.SIGNATURES) covers the whole header."""
    from beamtrace2007_b200 import _native as N
    missing = [n for n in _declared() if n not in N.SIGNATURES]
    assert not missing, missing


def test_no_device_is_an_error_not_an_abort(native_lib):
    """Without a GPU (this container) every device call returns a status."""
    from beamtrace2007_b200 import _native as N
    info = N.GpuInfo()
    rc = native_lib.bt_gpu_available(C.byref(info))
    assert rc in (N.BT_OK, -6)
    if rc != N.BT_OK:
        assert native_lib.bt_gpu_last_error()


def test_invalid_arguments_rejected(native_lib):
    from beamtrace2007_b200 import _native as N
    assert native_lib.bt_gpu_create(None, None, None, C.byref(C.c_void_p())) == -1
    assert native_lib.bt_gpu_soft(None, None, None, None, None, None, None, None, None) == -1
    assert native_lib.bt_gpu_destroy(None) == 0
    bad = np.array([[0, 1, 7]], np.uint32)
    pos = np.zeros((3, 3), np.float32)
    out = np.zeros((1, 3), np.uint32)
    f = np.zeros(4, np.float32)
    assert native_lib.bt_scene_finalize(N.ptr(pos), 3, N.ptr(bad), 1, N.ptr(out), N.ptr(f), N.ptr(f), N.ptr(f)) == -1
