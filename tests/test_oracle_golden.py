"""The oracle against the reference's own outputs (golden fixtures).

The fixtures were produced by the reference's CPU tools built from its
sources (tests/golden/make_golden.py). The oracle must reproduce every
operator apply to float32 rounding of the reference (<= 1e-6 relative L2).
"""

import numpy as np
import pytest

from conftest import golden, rel
from oracle import nufft_oracle as orc

OPS_TOL = 1e-6


def _op(g, periodic=False):
    img = g["img"]
    while img.ndim < 4:
        img = img[..., None]
    traj = g["traj"].real.reshape(3, -1, order="F")
    return orc.NufftOracle(traj, img.shape[:3], periodic=periodic, weights=g.get("pattern")), img


UNEVEN = [("nufft2d_n40", False), ("nufft2d_n40_periodic", True), ("nufft3d_n12", False)]


@pytest.mark.parametrize("name,periodic", [("nufft2d_n64", False), ("nufft2d_n64_periodic", True),
                                           ("nufft3d_n16", False), ("nufft2d_n32_coils3", False),
                                           ("nufft2d_n64_weights", False)] + UNEVEN)
def test_forward_adjoint(name, periodic):
    g = golden(name)
    o, img = _op(g, periodic)
    C = img.shape[3]
    fwd = o.forward(img)
    assert rel(fwd, g["fwd"].reshape(-1, C, order="F")) < OPS_TOL
    adj = o.adjoint(g["ksp"].reshape(-1, C, order="F"))
    assert rel(adj, g["adj"].reshape(img.shape, order="F")) < OPS_TOL


@pytest.mark.parametrize("name,periodic", [("nufft2d_n64", False), ("nufft2d_n64_periodic", True),
                                           ("nufft3d_n16", False), ("nufft2d_n64_weights", False)] + UNEVEN)
def test_toeplitz_normal_and_psf(name, periodic):
    g = golden(name)
    o, img = _op(g, periodic)
    assert rel(o.normal_toeplitz(img), g["normal"].reshape(img.shape, order="F")) < OPS_TOL
    assert rel(o.normal_explicit(img), g["normal_explicit"].reshape(img.shape, order="F")) < OPS_TOL
    # PSF: reference sub-grid s, index w  <->  centred 2N cell 2w + s
    psf = g["psf"]
    dims3 = img.shape[:3]
    nd = sum(1 for d in dims3 if d > 1)
    P = o.psf()
    sub = psf.reshape(dims3 + (2 ** nd,), order="F")
    rec = np.zeros(P.shape, dtype=np.complex128)
    for s in range(2 ** nd):
        sl = []
        b = s
        for d in dims3:
            if d > 1:
                sl.append(slice(b & 1, None, 2))
                b >>= 1
            else:
                sl.append(slice(None))
        rec[tuple(sl)] = sub[..., s]
    assert rel(P, rec) < OPS_TOL


def test_nufft_close_to_ndft():
    """The NUFFT approximates the exact NDFT (accuracy of KB w=6, os=2)."""
    g = golden("nufft2d_n64_periodic")
    o, img = _op(g, periodic=True)
    exact = orc.ndft_forward(g["traj"].real.reshape(3, -1, order="F"), img)
    assert rel(o.forward(img), exact) < 1e-4


@pytest.mark.parametrize("name", ["pics2d_n64_c4", "pics2d_n48_c3", "pics3d_n16_c2"])
def test_pics_few_iterations(name):
    """CG-SENSE at 5 iterations matches the reference's pics (float32 CG)."""
    g = golden(name)
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    y = g["ksp"].reshape(-1, C, order="F")
    x, sc = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=5, scaling=1.0)
    assert rel(x, g["x5_w1"].reshape(x.shape, order="F")) < 1e-5
    x, sc = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=5, scaling=1.0, toeplitz=False)
    assert rel(x, g["x5_w1_notoep"].reshape(x.shape, order="F")) < 1e-5


def test_pics_scaling_and_30_iterations():
    """30 iterations: float32 CG (reference) and float64 CG (oracle) drift
    apart through rounding (not converged: residual ~1e-3); the data scaling
    rule and the -S rescale are exact."""
    g = golden("pics2d_n64_c4")
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    y = g["ksp"].reshape(-1, C, order="F")
    x, sc = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=30)
    ref = g["x30"].reshape(x.shape, order="F")
    assert rel(x, ref) < 2e-2
    xs, sc2 = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=30, rescale=True)
    assert sc2 == sc
    # two reference runs differ slightly: its CPU gridding adds with OpenMP
    # atomics in a varying order (doc/performance.txt:67-69)
    assert rel(g["x30_rescale"], g["x30"] * sc) < 1e-4


@pytest.mark.parametrize("name", ["pics2d_n64_c4", "pics2d_n48_c3"])
def test_pics_30_iterations_with_float32_scalars(name):
    """With the CG scalars rounded to float32 as the reference stores them,
    30 unconverged iterations stay within 2e-4 of the reference's pics
    (measured 1.6e-4 and 1.2e-4; float64 scalars drift to 1e-2): the drift
    comes from the scalars, not from the float32 vectors."""
    g = golden(name)
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    y = g["ksp"].reshape(-1, C, order="F")
    x, _ = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=30, f32_scalars=True)
    ref = g["x30"].reshape(x.shape, order="F")
    assert rel(x, ref) < 2.5e-4
    x64, _ = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=30)
    assert rel(x64, ref) > 10 * rel(x, ref)


@pytest.mark.parametrize("key,kw", [("inv_m5", dict(maxiter=5)), ("inv_m5_l", dict(maxiter=5, lam=0.1)),
                                    ("inv_m5_c", dict(maxiter=5, precond=True)),
                                    ("inv_m5_c_l", dict(maxiter=5, precond=True, lam=0.1))])
def test_nufft_inverse_and_circulant_precond(key, kw):
    """bart nufft -i [-c] [-l]: CG on (P^-1)(N^H N + lam) x = (P^-1) N^H y."""
    g = golden("inverse2d_n32_coils3")
    o = orc.NufftOracle(g["traj"].real.reshape(3, -1, order="F"), (32, 32, 1))
    x = orc.nufft_inverse(o, g["ksp"].reshape(-1, 3, order="F"), **kw)
    assert rel(x, g[key].reshape(32, 32, 1, 3, order="F")) < 1e-5


@pytest.mark.parametrize("name", ["nudft2d_n24", "nudft2d_n16_coils2"])
def test_ndft_vs_reference_nudft(name):
    """The FP64 NDFT against the reference's direct DFT (bart nufft -s). The
    reference scales by all image dims, coils included, and forms its phases
    in float32 (linear_phase, src/num/filter.c:256-265)."""
    g = golden(name)
    img = g["img"]
    while img.ndim < 4:
        img = img[..., None]
    C = img.shape[3]
    traj = g["traj"].real.reshape(3, -1, order="F")
    s = 1.0 / np.sqrt(C)
    assert rel(orc.ndft_forward(traj, img) * s, g["fwd"].reshape(-1, C, order="F")) < 2e-5
    adj = orc.ndft_adjoint(traj, g["ksp"].reshape(-1, C, order="F"), img.shape[:3]) * s
    assert rel(adj, g["adj"].reshape(adj.shape, order="F")) < 2e-5


def test_padded_precond_beats_strang_on_the_oracle():
    """The padded-circulant preconditioner (precond 3) on the FP64 oracle:
    symmetric positive definite (PCG converges), and fewer PCG iterations to
    1e-4 than the reference's Strang circulant on a golden 2D problem."""
    g = golden("pics2d_n64_c4")
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    A = orc.SenseOracle(traj, g["sens"])
    b = A.adjoint(g["ksp"].reshape(-1, C, order="F"))
    b = b / orc.estimate_scaling_norm(b)
    op = A.nufft
    axes = orc._axes(op.dims3)
    tot = float(np.prod([op.dims3[a] for a in axes]))
    pre = orc.circulant_precond(op)[..., None]

    def strang(v):
        return np.fft.ifftn(np.fft.fftn(v, axes=axes) / pre, axes=axes) * tot

    pad = orc.padded_precond(op, 0.01)
    rng = np.random.default_rng(0)
    v = rng.standard_normal(b.shape) + 1j * rng.standard_normal(b.shape)
    w = rng.standard_normal(b.shape) + 1j * rng.standard_normal(b.shape)
    assert abs(np.vdot(w, pad(v)) - np.vdot(pad(w), v)) < 1e-10 * abs(np.vdot(w, pad(v)))   # self-adjoint
    assert np.vdot(v, pad(v)).real > 0
    x3, it3 = orc.pcg(A.normal, b, 0.01, pad)
    x1, it1 = orc.pcg(A.normal, b, 0.01, strang)
    assert orc.normal_residual(A, x3, b, 0.01) < 1.5e-4
    assert it3 < it1, (it3, it1)


ROLL_SIDES = (8, 12, 16, 40, 48, 64, 128, 256, 512)


def test_kb_table_bitwise():
    """The oracle's Kaiser-Bessel table (1001 floats) and per-axis roll-off
    are bit-identical to the reference's (kbtable tool: kb_init through
    rolloff_correction, src/noncart/grid.c:45-97, 536-556)."""
    g = golden("kb_table")
    assert orc.calc_beta(2.0, 6.0) == float(g["beta"])
    beta = orc.kernel_beta(2.0, 6.0)
    t = orc.kb_table(beta)
    assert t.shape == g["kb"].shape == (1001,)
    assert np.array_equal(t.view(np.uint32), g["kb"].view(np.uint32))
    assert abs(orc.bessel_i0(beta) / float(g["i0beta"]) - 1.0) < 2e-15   # a few float64 ulp
    for n in ROLL_SIDES:
        r = orc.rolloff_axis(n, 2.0, 6.0, beta).astype(np.float32)
        assert np.array_equal(r.view(np.uint32), g[f"roll_{n}"].view(np.uint32)), n


def test_kooshball_32_two_coils():
    """The 3D golden-means kooshball (32^3, 400 x 64, 2 coils): oracle forward,
    adjoint and Toeplitz normal against the reference's nufft / refnormal
    (inputs regenerated from the fixture's seed and checked by checksum)."""
    import hashlib
    from bart_b200 import synth
    g = golden("nufft3d_n32_c2")
    rng = np.random.default_rng(int(g["seed"]))
    traj = synth.kooshball_traj(32, 400)
    img = (rng.standard_normal((32, 32, 32, 2)) + 1j * rng.standard_normal((32, 32, 32, 2))).astype(np.complex64)
    ksp = (rng.standard_normal((1, 64, 400, 2)) + 1j * rng.standard_normal((1, 64, 400, 2))).astype(np.complex64)
    for a, key in ((img, "img_sha256"), (ksp, "ksp_sha256")):
        assert hashlib.sha256(np.ascontiguousarray(a).tobytes(order="F")).hexdigest() == str(g[key])
    o = orc.NufftOracle(traj.real.reshape(3, -1, order="F"), (32, 32, 32))
    assert rel(o.forward(img), g["fwd"].reshape(-1, 2, order="F")) < OPS_TOL
    assert rel(o.adjoint(ksp.reshape(-1, 2, order="F")), g["adj"].reshape(32, 32, 32, 2, order="F")) < OPS_TOL
    assert rel(o.normal_toeplitz(img), g["normal"].reshape(32, 32, 32, 2, order="F")) < OPS_TOL


def _basis_oracle(g):
    """BasisNufftOracle of a basis fixture and its image [X, Y, 1, C, K]."""
    tr = g["traj"].real
    T, K = g["basis"].shape[5], g["basis"].shape[6]
    if tr.ndim >= 6 and tr.shape[5] == T:
        trajs = [tr[..., 0, 0, t].reshape(3, -1, order="F") for t in range(T)]
    else:
        trajs = [tr.reshape(3, -1, order="F")]
    w = None
    if "pattern" in g:
        w = [g["pattern"][0, :, :, 0, 0, t].reshape(-1, order="F") for t in range(T)]
    img = g["img"]
    X, Y, C = img.shape[0], img.shape[1], img.shape[3]
    op = orc.BasisNufftOracle(trajs, (X, Y, 1), g["basis"].reshape(T, K, order="F"), w)
    return op, img.reshape(X, Y, 1, C, K, order="F"), (X, Y, C, K, T)


@pytest.mark.parametrize("name", ["nufft2d_n32_basis", "nufft2d_n32_basis_shared"])
def test_basis_forward_adjoint_normal(name):
    """nufft -B: forward, adjoint, Toeplitz and explicit normal with a
    temporal basis (per-frame trajectories; or a shared trajectory with a
    per-frame sampling pattern) against the reference."""
    g = golden(name)
    op, x, (X, Y, C, K, T) = _basis_oracle(g)
    assert rel(op.forward(x), g["fwd"].reshape(-1, C, T, order="F")) < OPS_TOL
    assert rel(op.adjoint(g["ksp"].reshape(-1, C, T, order="F")), g["adj"].reshape(x.shape, order="F")) < OPS_TOL
    assert rel(op.normal_toeplitz(x), g["normal"].reshape(x.shape, order="F")) < OPS_TOL
    assert rel(op.adjoint(op.forward(x)), g["normal_explicit"].reshape(x.shape, order="F")) < OPS_TOL


@pytest.mark.parametrize("name", ["nufft2d_n64_chain", "nufft2d_n64_chain_weights", "nufft3d_n16_chain"])
def test_chain_forward_adjoint(name):
    """nufft -o os (os != 2: the reference's chained NUFFT on a grid of
    lround(os N) cells) against the reference, for every os of the fixture.
    Bar 3e-6: the reference's float32 FFTs of the 80-, 96- and 24-point grids
    round more than its power-of-two ones (measured 1.0-1.1e-6)."""
    g = golden(name)
    img = g["img"]
    while img.ndim < 4:
        img = img[..., None]
    traj = g["traj"].real.reshape(3, -1, order="F")
    for i, os_ in enumerate(g["oss"]):
        op = orc.ChainNufftOracle(traj, img.shape[:3], float(os_), weights=g.get("pattern"))
        C = img.shape[3]
        assert rel(op.forward(img), g[f"fwd_{i}"].reshape(-1, C, order="F")) < 3e-6, os_
        assert rel(op.adjoint(g["ksp"].reshape(-1, C, order="F")), g[f"adj_{i}"].reshape(img.shape, order="F")) \
            < 3e-6, os_
