"""GPU NUFFT through the C ABI against the reference's outputs and the oracle.

Bar: relative L2 <= 1e-5 per operator apply (forward, adjoint, Toeplitz
normal, PSF), on the golden fixtures (reference outputs) and on fresh seeded
inputs against the oracle.
"""

import numpy as np
import pytest

from bart_b200 import synth
from bart_b200.nufft import NufftConf, nufft_create2
from conftest import golden, rel
from oracle import nufft_oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _dims(img_shape):
    s = list(img_shape) + [1] * (4 - len(img_shape))
    return s


def _plan(g, periodic=False, toeplitz=True):
    img = g["img"]
    cd = _dims(img.shape)
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], cd[3]]
    w = g.get("pattern")
    wd = None if w is None else list(w.shape)
    return nufft_create2(kd, cd, td, g["traj"], wd, w, conf=NufftConf(toeplitz=toeplitz, periodic=periodic)), cd, kd


# image sides that are not powers of two: grid DFTs by Bluestein's algorithm
UNEVEN = [("nufft2d_n40", False), ("nufft2d_n40_periodic", True), ("nufft3d_n12", False)]


@pytest.mark.parametrize("name,periodic", [("nufft2d_n64", False), ("nufft2d_n64_periodic", True),
                                           ("nufft3d_n16", False), ("nufft2d_n32_coils3", False),
                                           ("nufft2d_n64_weights", False)] + UNEVEN)
def test_forward_adjoint_vs_reference(name, periodic):
    g = golden(name)
    op, cd, kd = _plan(g, periodic, toeplitz=False)
    fwd = op.forward(g["img"].reshape(cd, order="F"))
    assert rel(fwd, g["fwd"]) < TOL
    adj = op.adjoint(g["ksp"].reshape(kd, order="F"))
    assert rel(adj, g["adj"]) < TOL
    op.free()


@pytest.mark.parametrize("name,periodic", [("nufft2d_n64", False), ("nufft2d_n64_periodic", True),
                                           ("nufft3d_n16", False), ("nufft2d_n64_weights", False)] + UNEVEN)
def test_toeplitz_normal_and_psf_vs_reference(name, periodic):
    g = golden(name)
    op, cd, kd = _plan(g, periodic, toeplitz=True)
    n = op.normal(g["img"].reshape(cd, order="F"))
    assert rel(n, g["normal"]) < TOL
    psf = op.psf()
    assert rel(psf, g["psf"].reshape(psf.shape, order="F")) < TOL
    op.free()
    op, cd, kd = _plan(g, periodic, toeplitz=False)
    n = op.normal(g["img"].reshape(cd, order="F"))     # explicit adjoint(forward)
    assert rel(n, g["normal_explicit"]) < TOL
    op.free()


def _basis_plan(g, toeplitz):
    w = g.get("pattern")
    return nufft_create2(list(g["fwd"].shape), list(g["img"].shape), list(g["traj"].shape), g["traj"],
                         None if w is None else list(w.shape), w, list(g["basis"].shape), g["basis"],
                         conf=NufftConf(toeplitz=toeplitz))


@pytest.mark.parametrize("name", ["nufft2d_n32_basis", "nufft2d_n32_basis_shared"])
def test_basis_vs_reference(name):
    """Subspace basis (nufft -B): forward, adjoint, block-Toeplitz normal and
    the explicit normal against the reference's outputs; frames with their
    own trajectories, or one trajectory with a per-frame sampling pattern."""
    g = golden(name)
    op = _basis_plan(g, toeplitz=True)
    cd, kd = list(g["img"].shape), list(g["fwd"].shape)
    assert rel(op.forward(g["img"]), g["fwd"]) < TOL
    assert rel(op.adjoint(g["ksp"].reshape(kd, order="F")), g["adj"]) < TOL
    assert rel(op.normal(g["img"]), g["normal"]) < TOL
    op.free()
    op = _basis_plan(g, toeplitz=False)
    assert rel(op.normal(g["img"].reshape(cd, order="F")), g["normal_explicit"]) < TOL
    op.free()


def test_basis_uneven_size_and_3d_vs_oracle():
    """The basis on a non-power-of-two side (Bluestein spectra, block PSF on
    the 2N grid) and in 3D, against the oracle."""
    rng = np.random.default_rng(41)
    T, K, C = 3, 2, 2
    for N, ndim, spokes in ((40, 2, 30), (12, 3, 60)):
        t = synth.radial_traj(N, spokes) if ndim == 2 else synth.kooshball_traj(N, spokes)
        S = t.shape[2] // T
        tf = np.stack([t[:, :, f * S:(f + 1) * S] for f in range(T)], axis=-1).reshape(3, t.shape[1], S, 1, 1, T,
                                                                                    order="F")
        B = (rng.standard_normal((1, 1, 1, 1, 1, T, K)) + 1j * rng.standard_normal((1, 1, 1, 1, 1, T, K))).astype(
            np.complex64)
        Z = N if ndim == 3 else 1
        cd = [N, N, Z, C, 1, 1, K]
        kd = [1, t.shape[1], S, C, 1, T]
        x = (rng.standard_normal(cd) + 1j * rng.standard_normal(cd)).astype(np.complex64)
        op = nufft_create2(kd, cd, list(tf.shape), tf, None, None, list(B.shape), B, conf=NufftConf(toeplitz=True))
        o = orc.BasisNufftOracle([tf[..., 0, 0, f].real.reshape(3, -1, order="F") for f in range(T)], (N, N, Z),
                                 B.reshape(T, K, order="F"))
        xo = x.reshape(N, N, Z, C, K, order="F")
        assert rel(op.forward(x), o.forward(xo)) < TOL, (N, ndim)
        assert rel(op.normal(x), o.normal_toeplitz(xo)) < TOL, (N, ndim)
        op.free()


@pytest.mark.parametrize("N,spokes,coils", [(128, 64, 1), (64, 40, 2), (256, 402, 1), (512, 100, 1),
                                            (66, 30, 2), (200, 64, 1), (318, 90, 1), (320, 40, 2)])
def test_2d_vs_oracle(N, spokes, coils):
    rng = np.random.default_rng(N + spokes)
    t = synth.radial_traj(N, spokes)
    img = (rng.standard_normal((N, N, 1, coils)) + 1j * rng.standard_normal((N, N, 1, coils))).astype(np.complex64)
    cd = [N, N, 1, coils]
    kd = [1, t.shape[1], t.shape[2], coils]
    op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=True))
    o = orc.NufftOracle(t.real.reshape(3, -1, order="F"), (N, N, 1))
    assert rel(op.forward(img), o.forward(img)) < TOL
    y = (rng.standard_normal((t.shape[1] * t.shape[2], coils)) + 1j * rng.standard_normal((t.shape[1] * t.shape[2], coils))).astype(np.complex64)
    assert rel(op.adjoint(y.reshape(kd, order="F")), o.adjoint(y)) < TOL
    assert rel(op.normal(img), o.normal_toeplitz(img)) < TOL
    op.free()


def test_3d_vs_oracle():
    rng = np.random.default_rng(5)
    N = 32
    t = synth.kooshball_traj(N, 300)
    img = (rng.standard_normal((N, N, N, 1)) + 1j * rng.standard_normal((N, N, N, 1))).astype(np.complex64)
    cd = [N, N, N, 1]
    kd = [1, t.shape[1], t.shape[2], 1]
    op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=True))
    o = orc.NufftOracle(t.real.reshape(3, -1, order="F"), (N, N, N))
    assert rel(op.forward(img), o.forward(img)) < TOL
    y = (rng.standard_normal(kd[1] * kd[2]) + 1j * rng.standard_normal(kd[1] * kd[2])).astype(np.complex64)
    assert rel(op.adjoint(y.reshape(kd, order="F")), o.adjoint(y[:, None])) < TOL
    assert rel(op.normal(img), o.normal_toeplitz(img)) < TOL
    op.free()


def test_device_and_host_pointers_agree(cuda):
    import torch
    g = golden("nufft2d_n64")
    op, cd, kd = _plan(g, toeplitz=False)
    x = g["img"].reshape(cd, order="F").astype(np.complex64)
    host = op.forward(x)
    xd = torch.from_numpy(np.asfortranarray(x).ravel(order="F")).to(cuda)
    dev = op.forward(xd)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), np.asarray(host).ravel(order="F"))
    op.free()


def test_adjointness_full_size():
    """<A x, y> = <x, A^H y> at the 256^2, 402x512 single-coil size."""
    rng = np.random.default_rng(11)
    t = synth.radial_traj(256, 402)
    cd = [256, 256, 1, 1]
    kd = [1, 512, 402, 1]
    op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=False))
    x = (rng.standard_normal(cd) + 1j * rng.standard_normal(cd)).astype(np.complex64)
    y = (rng.standard_normal(kd) + 1j * rng.standard_normal(kd)).astype(np.complex64)
    ax = np.asarray(op.forward(x)).astype(np.complex128)
    ay = np.asarray(op.adjoint(y)).astype(np.complex128)
    lhs = np.vdot(ax.ravel(order="F"), y.astype(np.complex128).ravel(order="F"))
    rhs = np.vdot(x.astype(np.complex128).ravel(order="F"), ay.ravel(order="F"))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    op.free()


def test_unsupported_options_fail_loudly():
    """Options outside what is built are refused with a status, not run: an
    oversampled grid of odd length (os 1.25 on 34 pixels: 42.5 -> 42 is even,
    on 30: 37.5 -> 38 even, on 26: 32.5 -> 33 odd), os beyond 4, odd image
    sides, deterministic gridding with os != 2."""
    from bart_b200._lib import BnufftError
    t = synth.radial_traj(32, 8)
    with pytest.raises(BnufftError):
        nufft_create2([1, 64, 8, 1], [26, 26, 1, 1], list(t.shape), t, conf=NufftConf(os=1.25))
    with pytest.raises(BnufftError):
        nufft_create2([1, 64, 8, 1], [32, 32, 1, 1], list(t.shape), t, conf=NufftConf(os=5.0))
    with pytest.raises(BnufftError):
        nufft_create2([1, 64, 8, 1], [33, 33, 1, 1], list(t.shape), t)
    with pytest.raises(BnufftError):
        nufft_create2([1, 64, 8, 1], [32, 32, 1, 1], list(t.shape), t, conf=NufftConf(os=1.5, deterministic=True))


@pytest.mark.parametrize("name,periodic", [("nufft2d_n64", False), ("nufft2d_n64_periodic", True),
                                           ("nufft3d_n16", False), ("nufft2d_n32_coils3", False)])
def test_deterministic_mode_vs_reference(name, periodic):
    """Fixed-order (atomic-free) gridding: same parity bar as the default."""
    g = golden(name)
    img = g["img"]
    cd = _dims(img.shape)
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], cd[3]]
    toep = "normal" in g
    op = nufft_create2(kd, cd, td, g["traj"], conf=NufftConf(toeplitz=toep, periodic=periodic, deterministic=True))
    assert rel(op.forward(img.reshape(cd, order="F")), g["fwd"]) < TOL
    assert rel(op.adjoint(g["ksp"].reshape(kd, order="F")), g["adj"]) < TOL
    if toep:
        assert rel(op.normal(img.reshape(cd, order="F")), g["normal"]) < TOL
    op.free()


def test_deterministic_mode_is_bit_identical():
    """Two plans, two adjoints (and PSFs) of the same data: identical bits."""
    rng = np.random.default_rng(9)
    t = synth.radial_traj(256, 402)
    kd = [1, 512, 402, 4]
    cd = [256, 256, 1, 4]
    y = (rng.standard_normal(kd) + 1j * rng.standard_normal(kd)).astype(np.complex64)
    outs = []
    for _ in range(2):
        op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=True, deterministic=True))
        outs.append((np.asarray(op.adjoint(y)).copy(), op.psf().copy()))
        op.free()
    assert np.array_equal(outs[0][0].view(np.uint32), outs[1][0].view(np.uint32))
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))


@pytest.mark.parametrize("key,kw", [("inv_m5", dict(maxiter=5)), ("inv_m5_l", dict(maxiter=5, lam=0.1)),
                                    ("inv_m5_c", dict(maxiter=5, precond=True)),
                                    ("inv_m5_c_l", dict(maxiter=5, precond=True, lam=0.1))])
def test_nufft_inverse_vs_reference(key, kw):
    """bart nufft -i [-c] [-l] -m5 on three coil images."""
    g = golden("inverse2d_n32_coils3")
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], 3]
    op = nufft_create2(kd, [32, 32, 1, 3], td, g["traj"], conf=NufftConf(toeplitz=True))
    x = op.inverse(g["ksp"].reshape(kd, order="F"), **kw)
    op.free()
    assert rel(x, g[key]) < TOL


def test_nufft_inverse_30_iterations_precond():
    g = golden("inverse2d_n32_coils3")
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], 3]
    op = nufft_create2(kd, [32, 32, 1, 3], td, g["traj"], conf=NufftConf(toeplitz=True))
    x = op.inverse(g["ksp"].reshape(kd, order="F"), maxiter=30, precond=True)
    op.free()
    assert rel(x, g["inv_m30_c"]) < 1e-3


def test_lowmem_matches_default():
    """--lowmem (one coil's grid at a time) gives the default's results
    (deterministic gridding: identical bits)."""
    rng = np.random.default_rng(21)
    N, C = 48, 3
    t = synth.radial_traj(N, 20)
    img = (rng.standard_normal((N, N, 1, C)) + 1j * rng.standard_normal((N, N, 1, C))).astype(np.complex64)
    cd, kd = [N, N, 1, C], [1, t.shape[1], t.shape[2], C]
    out = {}
    for low in (False, True):
        op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=True, lowmem=low, deterministic=True))
        k = np.asarray(op.forward(img))
        out[low] = (k, np.asarray(op.adjoint(k.reshape(kd, order="F"))), np.asarray(op.normal(img)))
        op.free()
    for a, b in zip(out[False], out[True]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("deterministic", [True, False])
def test_update_traj_equals_fresh_plan(deterministic):
    """nufft_update_traj (src/noncart/nufft.c:2041-2054): a plan created with
    one trajectory and updated to another gives the same forward, adjoint,
    Toeplitz normal and PSF as a plan created with the second one (bit for
    bit in the deterministic mode; with atomic gridding to float32 rounding),
    and those match the reference's outputs for that trajectory."""
    g = golden("nufft2d_n64")
    cd, td = [64, 64, 1, 1], list(g["traj"].shape)
    kd = [1, td[1], td[2], 1]
    other = synth.radial_traj(64, td[2]).reshape(td)        # uniform spacing, different angles
    other[0] *= 0.9
    conf = NufftConf(toeplitz=True, deterministic=deterministic)
    fresh = nufft_create2(kd, cd, td, g["traj"], conf=conf)
    upd = nufft_create2(kd, cd, td, other, conf=conf)
    x = g["img"].reshape(cd, order="F")
    y = g["ksp"].reshape(kd, order="F")
    before = np.asarray(upd.normal(x)).copy()
    upd.update_traj(g["traj"])
    outs = {}
    for name, op in (("fresh", fresh), ("upd", upd)):
        outs[name] = (np.asarray(op.forward(x)), np.asarray(op.adjoint(y)), np.asarray(op.normal(x)), op.psf())
    for a, b in zip(outs["fresh"], outs["upd"]):
        if deterministic:
            assert np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))
        else:
            assert rel(b, a) < 1e-6
    fwd, adj, nrm, psf = outs["upd"]
    assert rel(fwd, g["fwd"]) < TOL
    assert rel(adj, g["adj"]) < TOL
    assert rel(nrm, g["normal"]) < TOL
    assert rel(psf, g["psf"]) < TOL
    assert rel(before, g["normal"]) > 1e-2      # the PSF really followed the trajectory
    fresh.free()
    upd.free()


@pytest.mark.parametrize("N,spokes,coils,nd,periodic", [(256, 96, 16, 2, False), (256, 402, 1, 2, False),
                                                         (128, 64, 3, 2, False), (64, 40, 2, 2, True),
                                                         (40, 30, 6, 2, False), (32, 300, 8, 3, False),
                                                         (32, 200, 1, 3, True), (48, 300, 4, 3, False)])
def test_tiled_scatter_matches_atomic(N, spokes, coils, nd, periodic, monkeypatch):
    """The output-stationary adjoint gridding (tiles with register
    accumulation and plain stores; the default for 3D multi-coil problems,
    BNUFFT_GRIDDING=lines everywhere) against the global-atomic scatter
    (selected by an explicit bin edge) and the oracle, on 2D and 3D,
    periodic and not, single- and multi-coil problems, dense centres
    included."""
    rng = np.random.default_rng(N * 7 + coils)
    t = synth.radial_traj(N, spokes) if nd == 2 else synth.kooshball_traj(N, spokes)
    cd = [N, N, 1 if nd == 2 else N, coils]
    kd = [1, t.shape[1], t.shape[2], coils]
    y = (rng.standard_normal(kd) + 1j * rng.standard_normal(kd)).astype(np.complex64)
    outs = []
    monkeypatch.setenv("BNUFFT_GRIDDING", "lines")
    for b in (0, 32):
        op = nufft_create2(kd, cd, list(t.shape), t, conf=NufftConf(toeplitz=False, periodic=periodic, bin=b))
        outs.append(np.asarray(op.adjoint(y)))
        op.free()
    monkeypatch.delenv("BNUFFT_GRIDDING")
    assert rel(outs[0], outs[1]) < 1e-6
    o = orc.NufftOracle(t.real.reshape(3, -1, order="F"), tuple(cd[:3]), periodic=periodic)
    want = o.adjoint(y.reshape(-1, coils, order="F"))
    assert rel(outs[0], want.reshape(cd, order="F")) < TOL


@pytest.mark.parametrize("name", ["nufft2d_n64_chain", "nufft2d_n64_chain_weights", "nufft3d_n16_chain"])
def test_chain_vs_reference(name):
    """Oversampling other than 2 (nufft -o 1.25 / 1.5 / 2.5: the reference's
    chained NUFFT on a grid of lround(os N) cells, Bluestein transforms):
    forward, adjoint and the normal (adjoint of the forward, as the chain
    has no Toeplitz form) against the reference's outputs."""
    g = golden(name)
    cd = _dims(g["img"].shape)
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], cd[3]]
    w = g.get("pattern")
    for i, os_ in enumerate(g["oss"]):
        op = nufft_create2(kd, cd, td, g["traj"], None if w is None else list(w.shape), w,
                           conf=NufftConf(toeplitz=True, os=float(os_)))
        img = g["img"].reshape(cd, order="F")
        assert rel(op.forward(img), g[f"fwd_{i}"]) < TOL, os_
        assert rel(op.adjoint(g["ksp"].reshape(kd, order="F")), g[f"adj_{i}"]) < TOL, os_
        o = orc.ChainNufftOracle(g["traj"].real.reshape(3, -1, order="F"), cd[:3], float(os_), weights=w)
        assert rel(op.normal(img), o.adjoint(o.forward(img))) < TOL, os_
        op.free()


def test_cli_nufft_basis(tmp_path):
    """python -m bart_b200 nufft -B (forward, then adjoint with -x) on the
    basis fixture, as the reference's `bart nufft -B`."""
    from bart_b200.__main__ import main_nufft
    from bart_b200.cfl import readcfl, writecfl
    g = golden("nufft2d_n32_basis")
    for n in ("traj", "img", "ksp", "basis"):
        writecfl(str(tmp_path / n), g[n])
    p = lambda n: str(tmp_path / n)     # noqa: E731
    assert 0 == main_nufft(["-B", p("basis"), p("traj"), p("img"), p("k")])
    assert rel(readcfl(p("k")), g["fwd"]) < TOL
    assert 0 == main_nufft(["-a", "-B", p("basis"), "-x", "32:32:1", p("traj"), p("ksp"), p("a")])
    assert rel(readcfl(p("a")), g["adj"]) < TOL
