"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/qlgpu.h declares, and fails cleanly without a device."""
import ctypes
import os
import re

import pytest

from ql_dns_b200 import _capi
from ql_dns_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*(qlgpu_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    build()
    return ctypes.CDLL(_capi.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "qlgpu_step" in names and "qlgpu_create" in names
    assert set(_capi.EXPORTS) == set(names), set(_capi.EXPORTS) ^ set(names)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_params_struct_layout_matches_header():
    # 5 ints, 3 doubles (8-aligned), 5 doubles, 1 int, 1 double, 2 ints
    assert ctypes.sizeof(_capi.qlgpu_params) == 112
    assert _capi.qlgpu_params.L.offset == 24 and _capi.qlgpu_params.dt.offset == 96


def test_version_string(lib):
    lib.qlgpu_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.qlgpu_version()


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ql_dns_b200.params import mri_16x16_nz32
    L = _capi.load()
    h = ctypes.c_void_p()
    cp = _capi.to_c(mri_16x16_nz32())
    rc = L.qlgpu_create(ctypes.byref(cp), 0, ctypes.byref(h))
    assert rc == 5 and not h.value
    buf = ctypes.create_string_buffer(256)
    L.qlgpu_last_error(None, buf, 256)
    assert b"device" in buf.value


def test_invalid_parameters_rejected_before_device():
    from ql_dns_b200.params import mri_16x16_nz32
    L = _capi.load()
    h = ctypes.c_void_p()
    for bad, code in ((dict(NZ=48), 2), (dict(nx=7), 1), (dict(dt=-0.1), 2), (dict(nu=0.0), 1)):
        cp = _capi.to_c(mri_16x16_nz32(**bad))
        assert L.qlgpu_create(ctypes.byref(cp), 0, ctypes.byref(h)) == code, bad


def test_debug_library_exports_every_declared_symbol():
    # the QLGPU_DEBUG variant (index checks, guard zones) has the same C ABI
    lib_path = build(debug=True)
    dl = ctypes.CDLL(lib_path)
    for name in declared_functions():
        assert hasattr(dl, name), name
    assert dl.qlgpu_debug_build() == 1
    rl = ctypes.CDLL(_capi.LIB_PATH)
    assert rl.qlgpu_debug_build() == 0
