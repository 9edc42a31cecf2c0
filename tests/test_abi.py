"""The C-ABI library loads and exports every entry point include/bnufft.h declares.

Runs without a GPU: no compute call is made, except argument checks that
fail before touching the device.
"""

import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "bnufft.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bnufft_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["bnufft_create2", "bnufft_apply_forward", "bnufft_apply_adjoint", "bnufft_apply_normal",
              "bnufft_pics_create", "bnufft_pics_run", "bnufft_free", "bnufft_last_error"]:
        assert s in syms


def test_library_exports_all_declared():
    from bart_b200 import _lib
    from bart_b200.build import build
    build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_argument_errors_without_device():
    """Bad arguments are reported as status codes, not aborts."""
    from bart_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    d = _lib.dims_array([1] * 16)
    st = lib.bnufft_create2(ctypes.byref(h), 2, d, d, d, None, None, None, None, None, None, None)
    assert st == 1
    assert "trajectory" in lib.bnufft_last_error().decode()
    with pytest.raises(_lib.BnufftError):
        _lib.check(st)
