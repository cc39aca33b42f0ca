"""The C ABI library without a GPU: it loads, exports every symbol that
include/lbm_b200.h declares, and the pure-host entry points answer."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbm_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from b200lbm import _capi
    L = _capi.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(_capi.EXPORTED)


def test_footprint_is_host_only():
    from b200lbm import _capi
    L = _capi.lib()
    n = 256 ** 3
    b = L.lbm_footprint_bytes(256, 256, 256, _capi.STORE_F32)
    # populations in 8-cell blocks of 4-direction groups: 27 -> 28 and 7 -> 8 slots;
    # macro and tag arrays carry a 64-element tail pad
    blocks = (n + 7) // 8
    pad = 64
    assert b == 2 * (28 + 8) * 8 * blocks * 4 + 2 * 5 * (n + pad) * 4 + 2 * (n + pad) + 2 * n * 4
    b16 = L.lbm_footprint_bytes(256, 256, 256, _capi.STORE_F16)
    assert b16 < b
    assert L.lbm_footprint_bytes(2, 8, 8, 0) == 0


def test_bad_handle_arguments():
    from b200lbm import _capi
    L = _capi.lib()
    assert L.lbm_destroy(None) == _capi.ERR_ARG
    out = C.c_void_p()
    assert L.lbm_create(2, 8, 8, 0, 0, C.byref(out)) == _capi.ERR_ARG
    assert L.lbm_create(8, 8, 8, 9, 0, C.byref(out)) == _capi.ERR_ARG


def test_product_path_fails_loudly_without_library(tmp_path, monkeypatch):
    from b200lbm import _capi
    monkeypatch.setattr(_capi, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_capi, "_lib", None)
    with pytest.raises(ImportError):
        _capi.lib()


def test_nan_watchdog_argument_checks():
    from b200lbm import _capi
    L = _capi.lib()
    assert L.lbm_set_nan_watchdog(None, 1) == _capi.ERR_ARG
