"""The drop-in, compiled: the reference's own `nufft` and `pics` tools built
from its sources with their nufft_create2() call sites bound to the adapter
(oracle/refbuild/nufft_bnufft.c), which builds the reference's linop on the
library's C ABI. The reference's host code (option parsing, .cfl I/O, the
maps chain, data scaling, its CPU CG) then drives the GPU NUFFT through
lop_fun_t callbacks. Outputs are compared with the reference's own CPU
results on the golden fixtures: 1e-5 per operator apply, 1e-4 for
reconstructions.

The reference's `ecalib` is built the same way with its calib() call
bound to bnufft_calib (oracle/refbuild/calib_bnufft.c).

The binaries (oracle/_ref/bin/{nufft,pics,ecalib}_bnufft) are built by
`make -f oracle/refbuild/Makefile` after `python -m bart_b200.build`.
"""

import os
import subprocess
import tempfile

import numpy as np
import pytest

from bart_b200.cfl import readcfl, writecfl
from conftest import ROOT, golden, rel

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "bin")


def _tool(name):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{name} not built (make -f oracle/refbuild/Makefile)")
    return exe


def _run(d, exe, *args):
    r = subprocess.run([exe] + list(args), cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r


def test_dropin_nufft_forward_adjoint():
    exe = _tool("nufft_bnufft")
    g = golden("nufft2d_n64")
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), g["traj"])
        writecfl(os.path.join(d, "x"), g["img"])
        writecfl(os.path.join(d, "y"), g["ksp"])
        _run(d, exe, "t", "x", "k")
        _run(d, exe, "-a", "-x64:64:1", "t", "y", "a")
        assert rel(readcfl(os.path.join(d, "k")), g["fwd"]) < 1e-5
        assert rel(readcfl(os.path.join(d, "a")), g["adj"]) < 1e-5


def test_dropin_nufft_inverse():
    """bart nufft -i: the reference's lsqr/CG on the library's Toeplitz normal."""
    exe = _tool("nufft_bnufft")
    g = golden("inverse2d_n32_coils3")
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), g["traj"])
        writecfl(os.path.join(d, "k"), g["ksp"])
        for key, args in [("inv_m5", ["-m5"]), ("inv_m5_l", ["-m5", "-l0.1"])]:
            _run(d, exe, "-i", "-x32:32:1", *args, "t", "k", "o")
            assert rel(readcfl(os.path.join(d, "o")), g[key]) < 1e-5, key


@pytest.mark.parametrize("key,args,tol", [("x5_w1", ["-i5", "-w1"], 1e-5),
                                          ("x5_w1_notoep", ["-i5", "-w1", "--no-toeplitz"], 1e-5),
                                          ("x30", ["-i30"], 1e-4)])
def test_dropin_pics(key, args, tol):
    """bart pics -l2 -r0.01 -t: SENSE model, scaling and CG of the reference
    on the library's NUFFT linop (Toeplitz normal or forward/adjoint)."""
    exe = _tool("pics_bnufft")
    g = golden("pics2d_n64_c4")
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), g["traj"])
        writecfl(os.path.join(d, "s"), g["sens"])
        writecfl(os.path.join(d, "k"), g["ksp"])
        r = _run(d, exe, "-d4", "-l2", "-r0.01", *args, "-t", "t", "k", "s", "o")
        assert "libbnufft" in r.stderr + r.stdout      # the adapter built the NUFFT
        assert rel(readcfl(os.path.join(d, "o")), g[key]) < tol


def test_dropin_nufft_basis():
    """bart nufft -B (forward and adjoint with a temporal basis) on the
    library's NUFFT."""
    exe = _tool("nufft_bnufft")
    g = golden("nufft2d_n32_basis")
    with tempfile.TemporaryDirectory() as d:
        for n in ("traj", "img", "ksp", "basis"):
            writecfl(os.path.join(d, n), g[n])
        _run(d, exe, "-B", "basis", "traj", "img", "k")
        _run(d, exe, "-a", "-B", "basis", "-x32:32:1", "traj", "ksp", "a")
        assert rel(readcfl(os.path.join(d, "k")), g["fwd"]) < 1e-5
        assert rel(readcfl(os.path.join(d, "a")), g["adj"]) < 1e-5


def test_dropin_pics_basis():
    """bart pics -B (subspace reconstruction, tests/pics.mk's basis cases):
    the reference's SENSE model with the basis and its CG on the library's
    block-Toeplitz NUFFT, against its CPU output (orthonormal basis of 3
    over 4 frames, 10 iterations, automatic scaling; measured 2.4e-6)."""
    exe = _tool("pics_bnufft")
    g = golden("pics2d_n32_basis")
    with tempfile.TemporaryDirectory() as d:
        for n, k in (("t", "traj"), ("k", "ksp"), ("s", "sens"), ("b", "basis"), ("w", "pattern")):
            writecfl(os.path.join(d, n), g[k])
        r = _run(d, exe, "-d4", "-l2", "-r0.01", f"-i{int(g['iters'])}", "-B", "b", "-p", "w", "-t", "t",
                 "k", "s", "o")
        assert "libbnufft" in r.stderr + r.stdout
        assert rel(readcfl(os.path.join(d, "o")), g["out"]) < 1e-4


@pytest.mark.parametrize("opts", [["--zero-mem"], ["--no-precomp"], ["--lowmem"]])
def test_dropin_nufft_memory_modes(opts):
    """The reference's memory options of `bart nufft` (zero-overhead mode, no
    precomputed tables, low-mem mode) change how much it holds, not its
    results; on the library they give the same forward and adjoint."""
    exe = _tool("nufft_bnufft")
    g = golden("nufft2d_n64")
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), g["traj"])
        writecfl(os.path.join(d, "x"), g["img"])
        writecfl(os.path.join(d, "y"), g["ksp"])
        _run(d, exe, *opts, "t", "x", "k")
        _run(d, exe, *opts, "-a", "-x64:64:1", "t", "y", "a")
        assert rel(readcfl(os.path.join(d, "k")), g["fwd"]) < 1e-5
        assert rel(readcfl(os.path.join(d, "a")), g["adj"]) < 1e-5


@pytest.mark.parametrize("conf", ["real-psf,upper-triag-psf,compress-psf", "real-psf", "upper-triag-psf",
                                  "compress-psf", "decomposed-psf"])
def test_dropin_pics_basis_psf_storage(conf):
    """tests/linsub.mk:90-97: pics -B with the reference's PSF storage options
    (real part only, upper triangle of the coefficient pairs, compressed to
    the sampled cells, decomposed) reconstructs the same image."""
    exe = _tool("pics_bnufft")
    g = golden("pics2d_n32_basis")
    with tempfile.TemporaryDirectory() as d:
        for n, k in (("t", "traj"), ("k", "ksp"), ("s", "sens"), ("b", "basis"), ("w", "pattern")):
            writecfl(os.path.join(d, n), g[k])
        _run(d, exe, "-l2", "-r0.01", f"-i{int(g['iters'])}", "--nufft-conf", conf, "-B", "b", "-p", "w", "-t", "t",
             "k", "s", "o")
        assert rel(readcfl(os.path.join(d, "o")), g["out"]) < 1e-4


def test_dropin_nufft_oversampling():
    """bart nufft -o 1.5 / 1.25 (the reference's chained NUFFT for os != 2)
    through the adapter, which passes conf.os on."""
    exe = _tool("nufft_bnufft")
    g = golden("nufft2d_n64_chain")
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "t"), g["traj"])
        writecfl(os.path.join(d, "x"), g["img"])
        writecfl(os.path.join(d, "y"), g["ksp"])
        for i, o in enumerate(g["oss"]):
            _run(d, exe, "-o", str(o), "t", "x", "k")
            _run(d, exe, "-o", str(o), "-a", "-x64:64:1", "t", "y", "a")
            assert rel(readcfl(os.path.join(d, "k")), g[f"fwd_{i}"]) < 1e-5, o
            assert rel(readcfl(os.path.join(d, "a")), g[f"adj_{i}"]) < 1e-5, o


@pytest.mark.parametrize("name", ["ecalib2d_n64_c8", "ecalib2d_n64_c8_m3_soft", "ecalib2d_40x48_c20",
                                  "ecalib3d_n24_c4", "ecalib2d_n64_c8_I", "ecalib2d_50x45_c8_m6"])
def test_dropin_ecalib(name):
    """The reference's own ecalib (option parsing, .cfl I/O, its
    calibration-region extraction) with calib() bound to bnufft_calib
    (oracle/refbuild/calib_bnufft.c) writes the maps and eigenvalue maps of
    the reference's CPU ecalib: the principal map and its eigenvalues to
    1e-4, lower maps and theirs to 1e-3, up to the global sign the reference takes from its
    LAPACK."""
    from test_espirit_oracle import map_error
    exe = _tool("ecalib_bnufft")
    g = golden(name)
    with tempfile.TemporaryDirectory() as d:
        writecfl(os.path.join(d, "k"), g["ksp"])
        _run(d, exe, *[str(a) for a in g["args"]], "k", "s", "e")
        s, e = readcfl(os.path.join(d, "s")), readcfl(os.path.join(d, "e"))
    assert s.shape == g["sens"].shape and e.shape == g["emaps"].shape
    sh = s.shape[:5]
    s, e = s.reshape(sh, order="F"), e.reshape(sh[:3] + (1, sh[4]), order="F")
    rs = g["sens"].reshape(sh, order="F")
    re = g["emaps"].reshape(e.shape, order="F")
    for m in range(sh[4]):
        bar = 1e-4 if m == 0 else 1e-3
        assert rel(e[..., m], re[..., m]) < bar, (m, rel(e[..., m], re[..., m]))
        assert map_error(s[..., m], rs[..., m]) < bar, m
