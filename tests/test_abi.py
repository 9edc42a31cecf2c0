"""The C-ABI library loads and exports every entry point include/*.h declares.

Runs without a GPU: no compute call is made, except argument checks that
fail before touching the device.
"""

import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    src = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bnufft_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["bnufft_create2", "bnufft_apply_forward", "bnufft_apply_adjoint", "bnufft_apply_normal",
              "bnufft_pics_create", "bnufft_pics_run", "bnufft_free", "bnufft_last_error", "bnufft_ecalib",
              "bnufft_ecalib_dims", "bnufft_ecalib_defaults"]:
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


def test_ecalib_host_side_without_device():
    """The ESPIRiT defaults and output dimensions are host-only calls; bad
    arguments come back as status codes."""
    from bart_b200.espirit import EcalibConf, output_dims
    sd, ed = output_dims([64, 48, 1, 8], EcalibConf(maps=3))
    assert sd[:5] == [64, 48, 1, 8, 3] and ed[:5] == [64, 48, 1, 1, 3]
    sd, ed = output_dims([1, 48, 40, 4])
    assert sd[:5] == [1, 48, 40, 4, 2]
    from bart_b200 import _lib
    lib = _lib.load()
    c = EcalibConf().to_c()
    assert lib.bnufft_ecalib(ctypes.byref(c), 16, _lib.dims_array([8] * 16), None, None, None, None, None, None,
                             None) == 1


def test_kb_table_bitwise_library():
    """The library's own table builder (the one every plan and the
    allocation-free entry point upload) gives the reference's 1001 floats
    bit for bit, and its float64 roll-off rounds to the reference's float
    roll-off (kb_precompute / rolloff_correction, src/noncart/grid.c:86-97,
    536-556). Host-only calls: no GPU needed."""
    import numpy as np
    from bart_b200 import _lib
    from conftest import golden
    lib = _lib.load()
    g = golden("kb_table")
    beta = lib.bnufft_calc_beta(2.0, 6.0)
    assert beta == float(g["beta"])
    t = np.zeros(1001, dtype=np.float32)
    kb_beta = float(np.float32(beta))     # rolloff_correction passes beta as float to kb_init
    _lib.check(lib.bnufft_kb_precompute(kb_beta, 1000, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    assert np.array_equal(t.view(np.uint32), g["kb"].view(np.uint32))
    for n in (8, 12, 16, 40, 48, 64, 128, 256, 512):
        r = np.zeros(n, dtype=np.float64)
        _lib.check(lib.bnufft_rolloff_axis(2.0, 6.0, n, r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        assert np.array_equal(r.astype(np.float32).view(np.uint32), g[f"roll_{n}"].view(np.uint32)), n


def test_ecalib_argument_statuses_without_device():
    """bnufft_ecalib rejects bad inputs before any device work: options that
    are not built (2), more than 32 coils (2), more maps than coils (1), a
    MAPS dimension other than 1 (1), an image side below twice the kernel
    (1), a missing output (1)."""
    import numpy as np
    from bart_b200 import _lib
    from bart_b200.espirit import EcalibConf
    lib = _lib.load()
    buf = np.zeros(16, dtype=np.complex64)
    p = ctypes.c_void_p(buf.ctypes.data)

    def status(dims, conf, sens=p):
        d = _lib.dims_array(list(dims) + [1] * (16 - len(dims)))
        return lib.bnufft_ecalib(ctypes.byref(conf.to_c()), 16, d, p, sens, None, None, None, None, None)

    assert status([64, 64, 1, 8], EcalibConf(weighting=True)) == 2
    assert status([64, 64, 1, 8], EcalibConf(crop=-1.0)) == 2
    assert status([64, 64, 1, 33], EcalibConf()) == 2
    assert status([64, 64, 1, 2], EcalibConf(maps=3)) == 1
    assert status([64, 64, 1, 8, 2], EcalibConf()) == 1
    assert status([10, 64, 1, 8], EcalibConf()) == 1
    assert status([64, 64, 1, 8], EcalibConf(), sens=None) == 1
    assert "maps" in lib.bnufft_last_error().decode() or "arguments" in lib.bnufft_last_error().decode()


def test_calib_and_cg_argument_statuses_without_device():
    """bnufft_calib / bnufft_calone / bnufft_cg_* report bad arguments as
    status 1 before touching the device."""
    import numpy as np
    from bart_b200 import _lib
    from bart_b200.espirit import EcalibConf
    lib = _lib.load()
    buf = np.zeros(16, dtype=np.complex64)
    p = ctypes.c_void_p(buf.ctypes.data)
    c = EcalibConf().to_c()

    def d16(dims):
        return _lib.dims_array(list(dims) + [1] * (16 - len(dims)))

    # output coils differ from the calibration data's
    assert lib.bnufft_calib(ctypes.byref(c), 16, d16([64, 64, 1, 4, 2]), p, None, 0, None, d16([24, 24, 1, 8]), p,
                            None) == 1
    # calibration region smaller than the kernel
    assert lib.bnufft_calib(ctypes.byref(c), 16, d16([64, 64, 1, 8, 2]), p, None, 0, None, d16([4, 24, 1, 8]), p,
                            None) == 1
    # too few singular-value slots for the 6x6x8-column calibration matrix
    assert lib.bnufft_calib(ctypes.byref(c), 16, d16([64, 64, 1, 8, 2]), p, None, 5,
                            (ctypes.c_float * 5)(), d16([24, 24, 1, 8]), p, None) == 1
    assert lib.bnufft_calone(ctypes.byref(c), 16, d16([64, 64, 1, 8]), p, None, None, None, None, None) == 1
    h = ctypes.c_void_p()
    assert lib.bnufft_cg_create(ctypes.byref(h), 0, 0.01, 0.0, 0, None) == 1
    assert lib.bnufft_cg_create(ctypes.byref(h), 16, -1.0, 0.0, 0, None) == 1
    assert lib.bnufft_cg_update(None, p, p, p, p, None) == 1
    assert lib.bnufft_cg_status(None, None, None, None, None) == 1
